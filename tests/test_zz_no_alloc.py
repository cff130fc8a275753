"""The batched compress entry point that allocates nothing
(frsz2_batch_compress_static), called through the C ABI.

Some callers cannot allocate device memory when they compress: their
allocator already owns the GPU's memory, or the request path forbids a
cudaMalloc.  This entry point keeps its work list in a fixed device array of
the library instead of a plan.  It must produce exactly what the oracle and
the plan-based frsz2_batch_compress produce for the same arrays, call after
call: the shared array keeps the previous call's contents, which must not
leak into the next, and a call issued right behind another on the same
stream must wait for the earlier call's kernels before it rewrites the work
list.  This file sorts last so a run that stops at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import frsz_b200
import oracle
from frsz_b200 import BatchArray, BatchPlan, workloads
from frsz_b200._lib import BatchItemC

pytestmark = pytest.mark.gpu

# first call: 14 arrays over ten classes, plus arrays with their own launch
SPECS_A = ([(np.float32, n, b, 32) for n, b in ((1000, 8), (70_001, 12), (4096 * 5, 16), (33, 24), (300_000, 32))] +
           [(np.float64, n, b, 32) for n, b in ((2048 * 3 + 1, 8), (50_000, 12), (1, 16), (90_000, 24), (7777, 32))] +
           [(np.float64, 40_000, 21, 64), (np.float32, 12_345, 13, 128),
            (np.float64, 10_000, 16, 5),    # handled by its own launch
            (np.float64, 0, 16, 32)])
# second call: fewer arrays, other classes and block sizes
SPECS_B = [(np.float32, 9_000, 20, 32), (np.float64, 123_457, 20, 32), (np.float32, 65_536, 32, 256),
           (np.float64, 3_001, 7, 16)]


def specs_c(count=400, seed=3):
    """Third call: more arrays than the first (more than one upload launch
    of descriptors), sizes 1..20,000, random float types and widths."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        dtype = np.float64 if rng.random() < 0.5 else np.float32
        out.append((dtype, int(rng.integers(1, 20_000)), int(rng.choice([8, 11, 16, 21, 24, 32])),
                    int(rng.choice([32, 64]))))
    return out


def build(specs, seed, canary):
    xs, bufs = [], []
    for k, (dtype, n, bits, E) in enumerate(specs):
        xs.append(workloads.loguniform_np(n, dtype, seed=seed + k, lo=-15, hi=15))
        size = frsz_b200.compressed_size(dtype, bits, E, n)
        bufs.append(torch.full((size,), canary, dtype=torch.uint8, device="cuda"))
    return xs, [torch.from_numpy(x).cuda() for x in xs], bufs


def static_compress(specs, xs, bufs):
    items = (BatchItemC * len(specs))()
    for i, ((dtype, n, bits, E), x, b) in enumerate(zip(specs, xs, bufs)):
        items[i].dtype = frsz_b200.FRSZ2_DOUBLE if dtype == np.float64 else frsz_b200.FRSZ2_FLOAT
        items[i].bits, items[i].block_size, items[i].n = bits, E, n
        items[i].values = x.data_ptr()
        items[i].decompressed = None
        items[i].compressed = b.data_ptr()
    stream = torch.cuda.current_stream().cuda_stream
    rc = frsz_b200.lib().frsz2_batch_compress_static(items, len(specs), ctypes.c_void_p(stream))
    assert rc == 0, frsz_b200.lib().frsz2_last_error()


def test_static_back_to_back_calls_match_oracle_and_plan(cuda):
    calls = [(SPECS_A, 100, 0x5C), (SPECS_B, 200, 0xA3), (specs_c(), 300, 0x3E)]
    built = [build(specs, seed, canary) for specs, seed, canary in calls]
    torch.cuda.synchronize()
    # three calls in a row on one stream, no host synchronisation between them
    for (specs, _, _), (_, dx, bufs) in zip(calls, built):
        static_compress(specs, dx, bufs)
    torch.cuda.synchronize()
    for call, ((specs, _, canary), (hx, dx, bufs)) in enumerate(zip(calls, built)):
        for i, ((dtype, n, bits, E), x, b) in enumerate(zip(specs, hx, bufs)):
            want = oracle.compress(x, bits, E, canary=canary)
            assert np.array_equal(b.cpu().numpy(), want), f"call {call}: array {i} {specs[i]} differs from the oracle"
        # the plan-based batched compress gives the same bytes
        pbufs = [torch.full_like(b, canary) for b in bufs]
        plan = BatchPlan([BatchArray(values=x, compressed=b, bits=bits, block_size=E)
                          for (dtype, n, bits, E), x, b in zip(specs, dx, pbufs)])
        plan.compress()
        torch.cuda.synchronize()
        for i, (s, p) in enumerate(zip(bufs, pbufs)):
            assert torch.equal(s, p), f"call {call}: array {i} {specs[i]} differs from the plan's output"
        plan.close()


def test_static_repeat_after_larger_call(cuda):
    """A small call right after a large one: the work list prefix it rewrites
    is shorter than what the large call left in the array."""
    for specs, seed, canary in ((specs_c(600, seed=9), 400, 0x11), (SPECS_B, 500, 0x77)):
        hx, dx, bufs = build(specs, seed, canary)
        static_compress(specs, dx, bufs)
        torch.cuda.synchronize()
        for i, ((dtype, n, bits, E), x, b) in enumerate(zip(specs, hx, bufs)):
            assert np.array_equal(b.cpu().numpy(), oracle.compress(x, bits, E, canary=canary)), (seed, i, specs[i])


def test_static_rejects_oversized_batch(cuda):
    items = (BatchItemC * 4097)()
    rc = frsz_b200.lib().frsz2_batch_compress_static(items, 4097, None)
    assert rc == 2
    assert b"at most 4096" in frsz_b200.lib().frsz2_last_error()
