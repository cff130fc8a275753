"""Decompress of the unaligned compile-time widths under each of their launch
shapes (256- or 128-thread CTAs, with or without the register cap for 2048
resident threads per SM, chosen per width): many tiles, ragged tails, padded
blocks, blocks larger than a 128-thread tile (which take the 256-thread
tile), block-range slices, special values, all against the oracle bit for
bit."""
import os

import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import shard, workloads

pytestmark = pytest.mark.gpu

THREADS = min(16, os.cpu_count() or 1)


def values_of(y):
    return y.view(np.uint64 if y.dtype == np.float64 else np.uint32)


def check_decompress(x, bits, E):
    ref = oracle.compress(x, bits, E, threads=THREADS)
    want = oracle.decompress(ref, x.size, x.dtype, bits, E, threads=THREADS)
    got = frsz_b200.decompress(torch.from_numpy(ref).cuda(), x.size, x.dtype, bits, E).cpu().numpy()
    if not np.array_equal(values_of(got), values_of(want)):
        bad = np.nonzero(values_of(got) != values_of(want))[0]
        raise AssertionError(f"values differ at {bad[:6]} (of {bad.size}); {x.dtype} bits={bits} E={E} n={x.size}")


@pytest.mark.parametrize("bits", [4, 5, 13, 21, 27, 37, 51, 63])
def test_fp64_many_tiles(cuda, bits):
    # 2^23 + ragged values
    n = (1 << 23) + 1234
    x = workloads.loguniform_np(n, np.float64, seed=bits, lo=-300, hi=300)
    for E in (32, 64):
        check_decompress(x, bits, E)


@pytest.mark.parametrize("bits", [5, 7, 11, 13, 21, 31])
def test_fp32_many_tiles(cuda, bits):
    n = (1 << 24) + 4097
    x = workloads.loguniform_np(n, np.float32, seed=100 + bits, lo=-30, hi=30)
    for E in (32, 256):
        check_decompress(x, bits, E)


@pytest.mark.parametrize("dtype,bits,E", [(np.float64, 21, 4), (np.float64, 21, 8), (np.float64, 13, 16),
                                          (np.float64, 37, 32), (np.float32, 13, 8), (np.float32, 5, 16)])
def test_padded_blocks(cuda, dtype, bits, E):
    # E * bits not a multiple of the word width: blocks end in pad bits
    te = 2048 if dtype == np.float64 else 4096
    n = 3000 * te + 333
    x = workloads.loguniform_np(n, dtype, seed=bits * E, lo=-20, hi=20)
    check_decompress(x, bits, E)


@pytest.mark.parametrize("n", [1, 1023, 1024, 1025, 2048, 2049, 4095, 2 * 2048, 5 * 2048 - 1])
def test_one_to_few_tiles(cuda, n):
    # a tile or a few; tails of 0, 1 and 1023 values
    x = workloads.loguniform_np(n, np.float64, seed=n, lo=-300, hi=300)
    check_decompress(x, 21, 32)


@pytest.mark.parametrize("dtype,bits,E", [(np.float64, 21, 1024), (np.float64, 21, 2048), (np.float64, 37, 2048),
                                          (np.float32, 13, 2048), (np.float32, 7, 4096), (np.float32, 23, 4096)])
def test_blocks_beyond_small_tile(cuda, dtype, bits, E):
    # blocks of 2048 fp64 / 4096 fp32 values do not fit a 128-thread tile
    n = 37 * E + 5
    x = workloads.loguniform_np(n, dtype, seed=E + bits, lo=-30, hi=30)
    check_decompress(x, bits, E)


def test_special_values(cuda):
    # blocks outside the plain domain (tiny, huge, Inf / NaN, zeros)
    rng = np.random.default_rng(5)
    n = 1 << 22
    x = workloads.loguniform_np(n, np.float64, seed=5, lo=-300, hi=300)
    fi = np.finfo(np.float64)
    for b in rng.choice(n // 32, 4000, replace=False):
        sl = slice(b * 32, b * 32 + 32)
        k = b % 4
        if k == 0:
            x[sl] = rng.standard_normal(32) * float(fi.tiny)
        elif k == 1:
            x[sl] = np.where(rng.random(32) < 0.5, -0.0, 0.0)
        elif k == 2:
            x[sl] = rng.standard_normal(32) * float(fi.max) / 4
        else:
            x[b * 32 + 3] = np.inf if b % 8 == 3 else np.nan
    for bits in (13, 21, 45):
        check_decompress(x, bits, 32)


@pytest.mark.parametrize("b0", [0, 3, 8, 4096, 4099])
def test_block_range_slices(cuda, b0):
    # a rank's block range starting at block b0
    n = 2048 * 5000 + 17
    bits, E = 21, 32
    x = workloads.loguniform_np(n, np.float64, seed=b0, lo=-300, hi=300)
    ref = oracle.compress(x, bits, E, threads=THREADS)
    want = oracle.decompress(ref, n, np.float64, bits, E, threads=THREADS)
    nb = (n + E - 1) // E
    b1 = nb - 7
    d_ref = torch.from_numpy(ref).cuda()
    out = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
    view = out[b0 * E:]
    if view.data_ptr() % 32 != 0:
        pytest.skip("values view off the 32-byte layout")
    shard.decompress_shard(d_ref, n, np.float64, bits, E, b0, b1, view)
    got = out.cpu().numpy()
    lo, hi = b0 * E, min(n, b1 * E)
    assert np.array_equal(values_of(got[lo:hi]), values_of(want[lo:hi]))
    assert np.all(got[:lo] == 7.0) and np.all(got[hi:] == 7.0)
