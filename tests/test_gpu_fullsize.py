"""GPU parity at the benchmark's full sizes, whole buffer against the oracle
(as the reference's own GPU test compares the whole compressed buffer,
test/test_frsz_gpu.cu:347-359): every byte of the canary-prefilled
compressed buffer and every decoded bit pattern, for all six cases of the
2 GiB fp64 configuration (2^28 values, blocks of 32 and 64 at 16 / 21 / 32
bits) and the fp32 512^3 field.  Beside that, size-independent properties:
the per-block error bound on every value, determinism, and idempotence of
compress(decompress(compress(x)))."""
import os

import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import workloads

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
CANARY = 0xFF


def whole_buffer_check(x: torch.Tensor, buf: torch.Tensor, y: torch.Tensor, bits: int, E: int):
    """buf (prefilled with CANARY before the GPU compress) equals the oracle's
    canary-prefilled buffer byte for byte, and y equals the oracle's decode of
    it bit for bit."""
    n = x.numel()
    dtype = np.float32 if x.dtype == torch.float32 else np.float64
    xh = x.cpu().numpy()
    ref = oracle.compress(xh, bits, E, canary=CANARY, threads=THREADS)
    got = buf.cpu().numpy()
    assert got.size == ref.size
    if not np.array_equal(got, ref):
        bad = np.flatnonzero(got != ref)
        raise AssertionError(f"{bad.size} bytes differ, first at {bad[:8].tolist()} of {ref.size}")
    del got
    want = oracle.decompress(ref, n, dtype, bits, E, threads=THREADS)
    uint = np.uint64 if dtype == np.float64 else np.uint32
    yh = y.cpu().numpy()
    if not np.array_equal(yh.view(uint), want.view(uint)):
        bad = np.flatnonzero(yh.view(uint) != want.view(uint))
        raise AssertionError(f"{bad.size} decoded values differ, first at {bad[:8].tolist()}")


def bound_check(x: torch.Tensor, buf: torch.Tensor, y: torch.Tensor, bits: int, E: int):
    """|x - x_hat| <= max(2^(e_b - bits + 2), 2^(e_b - 31)) for every value;
    returns (max abs error, max rel error over nonzero x)."""
    n = x.numel()
    w = frsz_b200.word_bits(bits) // 8
    nb = -(-n // E)
    exps = buf[: nb * w].view({1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]).to(torch.float64)
    bound = torch.maximum(torch.exp2(exps - bits + 2), torch.exp2(exps - 31))
    worst = 0.0
    max_abs = 0.0
    max_rel = 0.0
    chunk = 1 << 24
    for s in range(0, n, chunk):
        xe = x[s:s + chunk].to(torch.float64)
        err = (xe - y[s:s + chunk].to(torch.float64)).abs()
        m = xe.numel()
        b = bound[s // E: (s + m + E - 1) // E].repeat_interleave(E)[: m]
        worst = max(worst, float((err - b).max()))
        max_abs = max(max_abs, float(err.max()))
        nz = xe != 0
        if bool(nz.any()):
            max_rel = max(max_rel, float((err[nz] / xe[nz].abs()).max()))
    assert worst <= 0.0, f"error bound exceeded by {worst}"
    return max_abs, max_rel


@pytest.mark.parametrize("bits,E", [(16, 32), (21, 32), (32, 32), (16, 64), (21, 64), (32, 64)])
def test_fp64_loguniform_full_size(cuda, bits, E):
    """2^28 fp64 values: random sign, 10^U(-30, 30), 1 % zeros, 0.1 % subnormals."""
    n = 1 << 28
    x = workloads.loguniform_cuda(n, torch.float64, seed=bits + E)
    size = frsz_b200.compressed_size(np.float64, bits, E, n)
    buf = torch.full((size,), CANARY, dtype=torch.uint8, device="cuda")
    frsz_b200.compress(x, bits, E, out=buf)
    y = frsz_b200.decompress(buf, n, np.float64, bits, E)
    torch.cuda.synchronize()
    whole_buffer_check(x, buf, y, bits, E)
    bound_check(x, buf, y, bits, E)
    # determinism and idempotence: compressing the decoded values again gives
    # the same buffer
    buf2 = torch.full_like(buf, CANARY)
    frsz_b200.compress(y, bits, E, out=buf2)
    torch.cuda.synchronize()
    assert torch.equal(buf, buf2)
    del x, y, buf, buf2
    torch.cuda.empty_cache()


def test_fp64_loguniform_ragged_length(cuda):
    """A length that is not a multiple of the block size or the kernels' tile:
    the partial last block writes only its words, whole buffer compared."""
    n, bits, E = (1 << 27) - 12345, 16, 64
    x = workloads.loguniform_cuda(n, torch.float64, seed=7)
    buf = torch.full((frsz_b200.compressed_size(np.float64, bits, E, n),), CANARY, dtype=torch.uint8, device="cuda")
    frsz_b200.compress(x, bits, E, out=buf)
    y = frsz_b200.decompress(buf, n, np.float64, bits, E)
    torch.cuda.synchronize()
    whole_buffer_check(x, buf, y, bits, E)
    del x, y, buf
    torch.cuda.empty_cache()


def test_fp32_sinusoid_field_full_size(cuda):
    """The fp32 512^3 field, E 32, 16 bits."""
    x = workloads.sinusoid_field_cuda(512, 512, 512, seed=42)
    n = x.numel()
    buf = torch.full((frsz_b200.compressed_size(np.float32, 16, 32, n),), CANARY, dtype=torch.uint8, device="cuda")
    frsz_b200.compress(x, 16, 32, out=buf)
    y = frsz_b200.decompress(buf, n, np.float32, 16, 32)
    torch.cuda.synchronize()
    whole_buffer_check(x, buf, y, 16, 32)
    max_abs, _ = bound_check(x, buf, y, 16, 32)
    assert max_abs < 2.0 ** (3 - 16 + 2)  # |x| < 8 here, so e_b <= 2
    buf2 = frsz_b200.compress(y, 16, 32)
    torch.cuda.synchronize()
    assert torch.equal(buf[frsz_b200.exponent_size(np.float32, 16, 32, n):],
                       buf2[frsz_b200.exponent_size(np.float32, 16, 32, n):])
    del x, y, buf, buf2
    torch.cuda.empty_cache()
