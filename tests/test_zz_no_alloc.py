"""The batched compress entry point that allocates nothing
(frsz2_batch_compress_static), called through the C ABI.

Some callers cannot allocate device memory when they compress: their
allocator already owns the GPU's memory, or the request path forbids a
cudaMalloc.  This entry point keeps its work list in a fixed device array of
the library instead of a plan.  It must produce exactly what the plan-based
frsz2_batch_compress produces for the same arrays, call after call (the
shared array keeps the previous call's contents, which must not leak into
the next).  This file sorts last so a run that stops at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import frsz_b200
from frsz_b200 import BatchArray, BatchPlan, workloads
from frsz_b200._lib import BatchItemC

pytestmark = pytest.mark.gpu

SPECS = ([(np.float32, n, b, 32) for n, b in ((1000, 8), (70_001, 12), (4096 * 5, 16), (33, 24), (300_000, 32))] +
         [(np.float64, n, b, 32) for n, b in ((2048 * 3 + 1, 8), (50_000, 12), (1, 16), (90_000, 24), (7777, 32))] +
         [(np.float64, 40_000, 21, 64), (np.float32, 12_345, 13, 128),
          (np.float64, 10_000, 16, 5),    # handled by its own launch
          (np.float64, 0, 16, 32)])


def build(seed, canary):
    xs, static_bufs, plan_bufs = [], [], []
    for k, (dtype, n, bits, E) in enumerate(SPECS):
        x = torch.from_numpy(workloads.loguniform_np(n, dtype, seed=seed + k, lo=-15, hi=15)).cuda()
        size = frsz_b200.compressed_size(dtype, bits, E, n)
        xs.append(x)
        static_bufs.append(torch.full((size,), canary, dtype=torch.uint8, device="cuda"))
        plan_bufs.append(torch.full((size,), canary, dtype=torch.uint8, device="cuda"))
    return xs, static_bufs, plan_bufs


def static_compress(xs, bufs):
    items = (BatchItemC * len(SPECS))()
    for i, ((dtype, n, bits, E), x, b) in enumerate(zip(SPECS, xs, bufs)):
        items[i].dtype = frsz_b200.FRSZ2_DOUBLE if dtype == np.float64 else frsz_b200.FRSZ2_FLOAT
        items[i].bits, items[i].block_size, items[i].n = bits, E, n
        items[i].values = x.data_ptr()
        items[i].decompressed = None
        items[i].compressed = b.data_ptr()
    stream = torch.cuda.current_stream().cuda_stream
    rc = frsz_b200.lib().frsz2_batch_compress_static(items, len(SPECS), ctypes.c_void_p(stream))
    assert rc == 0, frsz_b200.lib().frsz2_last_error()


def test_static_matches_plan_on_consecutive_calls(cuda):
    for call, (seed, canary) in enumerate(((100, 0x5C), (200, 0xA3))):
        xs, sbufs, pbufs = build(seed, canary)
        static_compress(xs, sbufs)
        plan = BatchPlan([BatchArray(values=x, compressed=b, bits=bits, block_size=E)
                          for (dtype, n, bits, E), x, b in zip(SPECS, xs, pbufs)])
        plan.compress()
        torch.cuda.synchronize()
        for i, (s, p) in enumerate(zip(sbufs, pbufs)):
            assert torch.equal(s, p), f"call {call}: array {i} {SPECS[i]} differs from the plan's output"
        plan.close()


def test_static_rejects_oversized_batch(cuda):
    items = (BatchItemC * 4097)()
    rc = frsz_b200.lib().frsz2_batch_compress_static(items, 4097, None)
    assert rc == 2
    assert b"at most 4096" in frsz_b200.lib().frsz2_last_error()
