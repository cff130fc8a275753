"""GPU parity at the benchmark's full sizes, through size-independent
properties: oracle spot checks of block ranges (blocks are independent, so any
block range compressed alone must reproduce the same exponents and words),
the per-block error bound on every value, determinism, and idempotence of
compress(decompress(compress(x)))."""
import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import workloads

pytestmark = pytest.mark.gpu


def spot_check(x: torch.Tensor, buf: torch.Tensor, y: torch.Tensor, bits: int, E: int, ranges: int = 12,
               blocks: int = 2048, seed: int = 0):
    n = x.numel()
    dtype = np.float32 if x.dtype == torch.float32 else np.float64
    w = frsz_b200.word_bits(bits) // 8
    nb = -(-n // E)
    exp_bytes = frsz_b200.exponent_size(dtype, bits, E, n)
    bb = -(-E * bits // (8 * w)) * w
    rng = np.random.default_rng(seed)
    starts = sorted(set([0, max(0, nb - blocks)] + [int(s) for s in rng.integers(0, max(1, nb - blocks), ranges)]))
    for b0 in starts:
        k = min(blocks, nb - b0)
        xs = x[b0 * E: min(n, (b0 + k) * E)].cpu().numpy()
        ref = oracle.compress(xs, bits, E, canary=0)
        rexp = ref[: k * w]
        rwords = ref[frsz_b200.exponent_size(dtype, bits, E, xs.size):]
        gexp = buf[b0 * w: (b0 + k) * w].cpu().numpy()
        gw = buf[exp_bytes + b0 * bb: exp_bytes + b0 * bb + rwords.size].cpu().numpy()
        if b0 + k == nb and n % E:
            # partial last block: only the written words are defined
            last = (n - (nb - 1) * E) * bits
            keep = (k - 1) * bb + (-(-last // (8 * w))) * w
            rwords, gw = rwords[:keep], gw[:keep]
        assert np.array_equal(gexp, rexp), f"exponents differ in blocks [{b0}, {b0 + k})"
        assert np.array_equal(gw, rwords), f"words differ in blocks [{b0}, {b0 + k})"
        ys = oracle.decompress(ref, xs.size, dtype, bits, E)
        assert np.array_equal(y[b0 * E: b0 * E + xs.size].cpu().numpy().view(np.uint8), ys.view(np.uint8))


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


@pytest.mark.parametrize("bits,E,n", [(21, 32, 1 << 28), (16, 64, (1 << 28) - 12345), (32, 32, 1 << 27)])
def test_fp64_loguniform_full_size(cuda, bits, E, n):
    """Config 3: fp64 2^28, random sign, 10^U(-30, 30), 1% zeros, 0.1% subnormals."""
    x = workloads.loguniform_cuda(n, torch.float64, seed=bits + E)
    size = frsz_b200.compressed_size(np.float64, bits, E, n)
    buf = torch.zeros(size, dtype=torch.uint8, device="cuda")
    frsz_b200.compress(x, bits, E, out=buf)
    y = frsz_b200.decompress(buf, n, np.float64, bits, E)
    torch.cuda.synchronize()
    spot_check(x, buf, y, bits, E)
    bound_check(x, buf, y, bits, E)
    # determinism and idempotence
    buf2 = torch.zeros_like(buf)
    frsz_b200.compress(y, bits, E, out=buf2)
    torch.cuda.synchronize()
    assert torch.equal(buf, buf2)
    del x, y, buf, buf2
    torch.cuda.empty_cache()


def test_fp32_sinusoid_field_full_size(cuda):
    """Config 2: fp32 512^3 field, E 32, 16 bits."""
    x = workloads.sinusoid_field_cuda(512, 512, 512, seed=42)
    n = x.numel()
    buf = frsz_b200.compress(x, 16, 32)
    y = frsz_b200.decompress(buf, n, np.float32, 16, 32)
    torch.cuda.synchronize()
    spot_check(x, buf, y, 16, 32)
    max_abs, _ = bound_check(x, buf, y, 16, 32)
    assert max_abs < 2.0 ** (3 - 16 + 2)  # |x| < 8 here, so e_b <= 2
    buf2 = frsz_b200.compress(y, 16, 32)
    torch.cuda.synchronize()
    assert torch.equal(buf[frsz_b200.exponent_size(np.float32, 16, 32, n):],
                       buf2[frsz_b200.exponent_size(np.float32, 16, 32, n):])
    del x, y, buf, buf2
    torch.cuda.empty_cache()
