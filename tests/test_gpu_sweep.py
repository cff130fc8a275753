"""GPU parity sweeps over every compile-time width, every block-size path
and special values (NaN, +-Inf, -0, subnormals, tiny / huge block
exponents), kernel against the oracle, whole buffers bit-exact."""
import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import workloads

pytestmark = pytest.mark.gpu


def run(x, bits, E, canary=0x6B):
    size = frsz_b200.compressed_size(x.dtype, bits, E, x.size)
    buf = torch.full((size,), canary, dtype=torch.uint8, device="cuda")
    frsz_b200.compress(torch.from_numpy(x).cuda(), bits, E, out=buf)
    got = buf.cpu().numpy()
    ref = oracle.compress(x, bits, E, canary=canary)
    y = frsz_b200.decompress(torch.from_numpy(ref).cuda(), x.size, x.dtype, bits, E).cpu().numpy()
    yr = oracle.decompress(ref, x.size, x.dtype, bits, E)
    return got, ref, y, yr


def check(x, bits, E):
    got, ref, y, yr = run(x, bits, E)
    if not np.array_equal(got, ref):
        bad = np.nonzero(got != ref)[0]
        raise AssertionError(f"compressed bytes differ at {bad[:6]} (of {bad.size}); bits={bits} E={E} n={x.size}")
    if not np.array_equal(y.view(np.uint8), yr.view(np.uint8)):
        bad = np.nonzero(y.view(np.uint64 if y.dtype == np.float64 else np.uint32) !=
                         yr.view(np.uint64 if y.dtype == np.float64 else np.uint32))[0]
        raise AssertionError(f"values differ at {bad[:6]} (of {bad.size}); bits={bits} E={E} n={x.size}")


@pytest.mark.parametrize("bits", range(4, 33))
def test_fp32_every_width(cuda, bits):
    for E, n in ((32, 3 * 4096 + 77), (8, 4096 + 5), (256, 2 * 4096),
                 # blocks smaller than a lane's 8 values
                 (4, 2 * 4096 + 5), (2, 4096 + 13), (1, 4096 + 1)):
        check(workloads.loguniform_np(n, np.float32, seed=bits * 7 + E, lo=-30, hi=30), bits, E)


@pytest.mark.parametrize("bits", range(4, 65))
def test_fp64_every_width(cuda, bits):
    lo, hi = (-30, 30) if bits <= 8 else (-300, 300)
    for E, n in ((32, 3 * 2048 + 77), (4, 2048 + 3), (128, 2 * 2048 + 1),
                 # blocks smaller than a lane's 4 values
                 (2, 2 * 2048 + 7), (1, 2048 + 5)):
        check(workloads.loguniform_np(n, np.float64, seed=bits * 11 + E, lo=lo, hi=hi), bits, E)


@pytest.mark.parametrize("dtype,E", [(np.float32, e) for e in (8, 16, 64, 128, 512, 1024, 2048, 4096)] +
                         [(np.float64, e) for e in (4, 8, 16, 64, 256, 512, 1024, 2048)])
def test_block_sizes(cuda, dtype, E):
    # 28 (fp32) and 56 (fp64) bits: seven-word lane segments staged through shared memory
    for bits in (8, 12, 16, 21, 24, 28, 32) + ((40, 56, 64) if dtype == np.float64 else ()):
        n = 5 * (4096 if dtype == np.float32 else 2048) + 3 * E // 2 + 1
        check(workloads.loguniform_np(n, dtype, seed=E + bits, lo=-20, hi=20), bits, E)


@pytest.mark.parametrize("dtype,E", [(np.float32, e) for e in (24, 40, 48, 56, 72, 96, 120, 1000, 12, 20, 100)] +
                         [(np.float64, e) for e in (12, 20, 24, 36, 48, 100, 1000, 2044, 6, 10, 18, 102)])
def test_block_sizes_multiple_of_a_lane(cuda, dtype, E):
    """Block sizes that are a multiple of a lane's values, or of half of them
    (fp32 12 / 20 / 100, fp64 6 / 10 / 18 / 102: decompress only), but not a
    power of two: whole-block tiles (padded blocks at 13, 21, 33 and 37 bits:
    decompress only), with a partial last block and a partial last tile."""
    te = 4096 if dtype == np.float32 else 2048
    for bits in (8, 12, 13, 16, 20, 21, 24, 32) + ((33, 37, 40, 48, 64) if dtype == np.float64 else ()):
        n = 3 * te + 7 * E // 2 + 5
        check(workloads.loguniform_np(n, dtype, seed=3 * E + bits, lo=-20, hi=20), bits, E)


def special_values(dtype, n, seed):
    rng = np.random.default_rng(seed)
    fi = np.finfo(dtype)
    x = workloads.loguniform_np(n, dtype, seed, lo=-5, hi=5)
    # whole blocks at the edges of the exponent range
    B = 64
    nb = n // B
    for b in rng.choice(nb, nb // 4, replace=False):
        kind = rng.integers(5)
        sl = slice(b * B, (b + 1) * B)
        if kind == 0:    # tiny: block exponent far below the plain range
            x[sl] = (rng.standard_normal(B) * float(fi.tiny) * 2 ** rng.integers(0, 40)).astype(dtype)
        elif kind == 1:  # only subnormals and zeros
            x[sl] = (rng.random(B) * float(fi.tiny)).astype(dtype) * (rng.random(B) < 0.7)
        elif kind == 2:  # near the top of the range (the largest overflow to +-Inf)
            with np.errstate(over="ignore"):
                x[sl] = (rng.standard_normal(B) * float(fi.max) / 4).astype(dtype)
        elif kind == 3:  # signed zeros
            x[sl] = np.where(rng.random(B) < 0.5, -0.0, 0.0).astype(dtype)
        else:            # exponent boundary of the plain range
            e = -95 if dtype == np.float32 else -959
            x[sl] = (rng.standard_normal(B) * 2.0 ** e).astype(dtype)
    return x


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_special_values(cuda, dtype):
    x = special_values(dtype, 64 * 512 + 13, 5)
    widths = (4, 8, 9, 16, 21, 24, 31, 32) if dtype == np.float32 else (4, 5, 7, 8, 9, 16, 21, 32, 33, 47, 63, 64)
    small = (1, 2, 4) if dtype == np.float32 else (1, 2)
    for bits in widths:
        for E in (8, 32, 64) + small:
            check(x, bits, E)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_nan_inf(cuda, dtype):
    """NaN is skipped by the block max (std::max); +-Inf blocks follow the
    oracle's definition of the reference's out-of-range shifts."""
    rng = np.random.default_rng(9)
    n = 4096 * 3 + 5
    x = workloads.normal_np(n, dtype, 3)
    x[rng.choice(n, 40, replace=False)] = np.nan
    x[rng.choice(n, 10, replace=False)] = np.inf
    x[rng.choice(n, 10, replace=False)] = -np.inf
    for bits in ((8, 16, 21, 32) if dtype == np.float32 else (8, 16, 21, 32, 40, 64)):
        # 24, 48 (and 20: half a lane for fp32): block sizes that are not powers of
        # two, with block maxima through shared memory; 128 / 256 / 512: blocks of
        # one or two warp rows, maxima by warp reductions
        for E in (8, 32, 24, 48, 20, 128, 256, 512):
            check(x, bits, E)


@pytest.mark.parametrize("E", [3, 5, 6, 7, 12, 48, 100, 257, 1000, 2047])
def test_block_sizes_not_powers_of_two(cuda, E):
    """Block sizes that are not powers of two (one-thread-per-block kernels up
    to 16, whole-block tiles of the fast kernels for multiples of a lane's
    values, chunked and warp-per-block kernels for the rest): several chunks,
    a partial last block, special values."""
    for dtype, widths in ((np.float32, (4, 9, 16, 21, 32)), (np.float64, (5, 8, 21, 33, 52, 64))):
        n = 3 * 2048 + 2 * E + E // 2 + 1
        x = special_values(dtype, n, E)
        for bits in widths:
            check(x, bits, E)


@pytest.mark.parametrize("dtype,bits", [(np.float32, b) for b in range(4, 33)] + [(np.float64, b) for b in range(4, 65)])
def test_small_blocks_every_width(cuda, dtype, bits):
    """The one-thread-per-block kernels (block sizes up to 16 that the fast
    kernels do not take): every width, block sizes 3, 5, 11 and 16 (16 with
    the values off the 32-byte layout), several chunks of whole blocks, a
    partial last block, special values."""
    es = np.dtype(dtype).itemsize
    for E in (3, 5, 11, 16):
        n = (5 * 4096 if es == 4 else 5 * 2048) + 2 * E + E // 2 + 1
        x = special_values(dtype, n, bits * 31 + E)
        if E != 16:
            check(x, bits, E)
            continue
        tv = torch.zeros(n + 1, dtype=torch.float32 if es == 4 else torch.float64, device="cuda")
        tv[1:] = torch.from_numpy(x).cuda()
        size = frsz_b200.compressed_size(dtype, bits, E, n)
        buf = torch.full((size,), 0x33, dtype=torch.uint8, device="cuda")
        frsz_b200.compress(tv[1:], bits, E, out=buf)
        ref = oracle.compress(x, bits, E, canary=0x33)
        assert np.array_equal(buf.cpu().numpy(), ref), (bits, E)
        out = torch.zeros(n + 1, dtype=tv.dtype, device="cuda")
        frsz_b200.decompress(torch.from_numpy(ref).cuda(), n, dtype, bits, E, out=out[1:])
        uint = np.uint64 if es == 8 else np.uint32
        assert np.array_equal(out[1:].cpu().numpy().view(uint), oracle.decompress(ref, n, dtype, bits, E).view(uint))


@pytest.mark.parametrize("dtype,bits", [(np.float32, b) for b in range(4, 33)] + [(np.float64, b) for b in range(4, 33)])
def test_blocks_17_to_64_every_width(cuda, dtype, bits):
    """Block sizes 17..64 that are not powers of two with 16-byte block
    starts (compress on the blockvec kernel: block bytes a multiple of 16 or
    only of 4, the partial last block on the generic kernel; decompress on
    the chunked kernel), special values."""
    Es = (20, 24, 36, 44, 48, 60) if dtype == np.float32 else (18, 22, 24, 34, 48, 62)
    for E in Es:
        n = 700 * E + E // 3 + 1
        x = special_values(dtype, n, bits * 13 + E)
        check(x, bits, E)


@pytest.mark.parametrize("dtype,bits", [(np.float32, b) for b in range(4, 33)] + [(np.float64, b) for b in range(4, 65)])
def test_values_off_32_bytes_every_width(cuda, dtype, bits):
    """Values pointer 1..7 (fp32) or 1..3 (fp64) elements past a 32-byte
    boundary with a 32-byte aligned buffer (the fast kernels' MIS instances):
    several whole tiles, a partial last tile, special values; bytes and values
    equal the oracle's, and decompress writes nothing outside its output."""
    es = np.dtype(dtype).itemsize
    P = 32 // es
    tdt = torch.float32 if es == 4 else torch.float64
    uint = np.uint32 if es == 4 else np.uint64
    for E in (P, 32, 256):
        k = 1 + (bits + E) % (P - 1)
        n = (3 * 4096 if es == 4 else 3 * 2048) + 3 * E + 5
        x = special_values(dtype, n, bits * 7 + E)
        base = torch.zeros(n + 2 * P, dtype=tdt, device="cuda")
        base[k:k + n] = torch.from_numpy(x).cuda()
        size = frsz_b200.compressed_size(dtype, bits, E, n)
        buf = torch.full((size,), 0x21, dtype=torch.uint8, device="cuda")
        frsz_b200.compress(base[k:k + n], bits, E, out=buf)
        ref = oracle.compress(x, bits, E, canary=0x21)
        assert np.array_equal(buf.cpu().numpy(), ref), (bits, E, k)
        out = torch.full((n + 2 * P,), -7.0, dtype=tdt, device="cuda")
        frsz_b200.decompress(torch.from_numpy(ref).cuda(), n, dtype, bits, E, out=out[k:k + n])
        got = out.cpu().numpy()
        want = oracle.decompress(ref, n, dtype, bits, E)
        assert np.array_equal(got[k:k + n].view(uint), want.view(uint)), (bits, E, k)
        assert np.all(got[:k] == -7.0) and np.all(got[k + n:] == -7.0), (bits, E, k)


@pytest.mark.parametrize("dtype,bits,E", [(np.float32, 16, 32), (np.float32, 21, 8), (np.float64, 40, 4),
                                          (np.float64, 21, 64), (np.float32, 13, 1)])
def test_pointers_off_alignment(cuda, dtype, bits, E):
    """Values and buffers at 4- and 8-byte offsets from 32-byte alignment
    (not the fast kernels' layout): bytes and values still match the oracle,
    bytes outside the buffer untouched."""
    n = 2 * 4096 + 3 * E + 5
    x = workloads.loguniform_np(n, dtype, seed=bits + E, lo=-20, hi=20)
    es = np.dtype(dtype).itemsize
    size = frsz_b200.compressed_size(dtype, bits, E, n)
    w = frsz_b200.word_bits(bits) // 8  # the buffer must be word aligned
    for voff, boff in ((1, w), (3, 3 * w), (2, 5 * w)):
        tv = torch.zeros(n + 4, dtype=torch.float32 if dtype == np.float32 else torch.float64, device="cuda")
        tv[voff:voff + n] = torch.from_numpy(x).cuda()
        raw = torch.full((size + 64,), 0x5A, dtype=torch.uint8, device="cuda")
        buf = raw[boff:boff + size]
        frsz_b200.compress(tv[voff:voff + n], bits, E, out=buf)
        ref = oracle.compress(x, bits, E, canary=0x5A)
        assert np.array_equal(buf.cpu().numpy(), ref), (voff, boff)
        assert np.all(raw[:boff].cpu().numpy() == 0x5A) and np.all(raw[boff + size:].cpu().numpy() == 0x5A)
        y = torch.zeros_like(tv)
        frsz_b200.decompress(buf, n, dtype, bits, E, out=y[voff:voff + n])
        want = oracle.decompress(ref, n, dtype, bits, E)
        uint = np.uint64 if dtype == np.float64 else np.uint32
        assert np.array_equal(y[voff:voff + n].cpu().numpy().view(uint), want.view(uint)), (voff, boff)


@pytest.mark.parametrize("dtype,bits", [(np.float32, b) for b in range(4, 33)] + [(np.float64, b) for b in range(4, 65)])
def test_compile_time_block_sizes_every_width(cuda, dtype, bits):
    """Block sizes 6, 7 and 12, which have compile-time instances (as 3 and
    5 do, above): every width, several chunks of whole blocks, a partial
    last block, special values."""
    es = np.dtype(dtype).itemsize
    for E in (6, 7, 12):
        n = (5 * 4096 if es == 4 else 5 * 2048) + 3 * E + E // 2 + 1
        check(special_values(dtype, n, bits * 17 + E), bits, E)


@pytest.mark.parametrize("E", [3, 5, 6, 7, 12])
def test_compile_time_block_sizes_off_alignment(cuda, E):
    """Values and buffers off 16-byte boundaries on the compile-time block
    sizes: bytes and values equal the oracle's, nothing written outside."""
    for dtype, bits in ((np.float32, 9), (np.float32, 16), (np.float32, 21), (np.float64, 9), (np.float64, 33)):
        es = np.dtype(dtype).itemsize
        n = 3 * 4096 + 2 * E + 1
        x = special_values(dtype, n, bits + E)
        size = frsz_b200.compressed_size(dtype, bits, E, n)
        w = frsz_b200.word_bits(bits) // 8
        tdt = torch.float32 if es == 4 else torch.float64
        uint = np.uint32 if es == 4 else np.uint64
        for voff, boff in ((1, w), (3, 3 * w)):
            tv = torch.zeros(n + 4, dtype=tdt, device="cuda")
            tv[voff:voff + n] = torch.from_numpy(x).cuda()
            raw = torch.full((size + 64,), 0x5A, dtype=torch.uint8, device="cuda")
            buf = raw[boff:boff + size]
            frsz_b200.compress(tv[voff:voff + n], bits, E, out=buf)
            ref = oracle.compress(x, bits, E, canary=0x5A)
            assert np.array_equal(buf.cpu().numpy(), ref), (dtype, bits, voff, boff)
            r = raw.cpu().numpy()
            assert np.all(r[:boff] == 0x5A) and np.all(r[boff + size:] == 0x5A)
            y = torch.full((n + 4,), -7.0, dtype=tdt, device="cuda")
            frsz_b200.decompress(buf, n, dtype, bits, E, out=y[voff:voff + n])
            got = y.cpu().numpy()
            want = oracle.decompress(ref, n, dtype, bits, E)
            assert np.array_equal(got[voff:voff + n].view(uint), want.view(uint)), (dtype, bits, voff, boff)
            assert np.all(got[:voff] == -7.0) and np.all(got[voff + n:] == -7.0)


def top_of_range_values(dtype, n, seed):
    """Blocks of 32 whose values have every mantissa bit set (and their
    neighbours one ulp down), at random exponents across the plain range and
    random signs, mixed with zeros, subnormals and values far below the block
    maximum: the codes reach 2^(bits-1) - 1, the largest magnitude the plain
    range encodes."""
    rng = np.random.default_rng(seed)
    fi = np.finfo(dtype)
    ones = dtype(2.0) - fi.eps  # 1.111...1 in binary
    lo, hi = (-90, 120) if dtype == np.float32 else (-950, 1000)
    x = np.empty(n, dtype=dtype)
    for b in range(0, n, 32):
        e = int(rng.integers(lo, hi))
        blk = (ones * np.power(dtype(2.0), dtype(e))).astype(dtype) * np.ones(32, dtype=dtype)
        blk[1::3] = np.nextafter(blk[1::3], dtype(0))
        blk[2::5] = blk[2::5] * dtype(2.0) ** -int(rng.integers(1, 40))
        blk[3] = 0.0
        blk[4] = float(fi.tiny) * 0.5 if e > lo + 40 else blk[4]
        blk *= np.where(rng.random(32) < 0.5, -1, 1).astype(dtype)
        x[b:b + 32] = blk[: min(32, n - b)]
    return x


@pytest.mark.parametrize("dtype,bits", [(np.float32, b) for b in (4, 8, 13, 16, 23, 24, 25, 32)] +
                         [(np.float64, b) for b in (4, 16, 31, 32, 33, 52, 53, 54, 64)])
def test_plain_range_top_codes(cuda, dtype, bits):
    """The largest magnitudes of the plain range (codes up to 2^(bits-1) - 1)
    on the fast and the blockwise kernels, around the widths where the
    fused multiply-add truncation stops (24 for fp32, 53 for fp64)."""
    n = 4 * 4096 + 77
    x = top_of_range_values(dtype, n, bits)
    for E in (32, 5, 8):
        check(x, bits, E)


@pytest.mark.parametrize("dtype,bits", [(np.float32, b) for b in range(4, 33)] + [(np.float64, b) for b in range(4, 65)])
def test_blocks_17_to_128_every_width(cuda, dtype, bits):
    """Block sizes 17..128 that are not powers of two (the compile-time-width
    chunked kernels): several chunks, a partial last block, special values,
    values pointers off 16-byte alignment; compressed bytes equal the
    oracle's, nothing written outside the buffer or the output."""
    es = np.dtype(dtype).itemsize
    tdt = torch.float32 if es == 4 else torch.float64
    uint = np.uint32 if es == 4 else np.uint64
    for E in (17, 33, 100, 128 - (bits % 3)):
        n = 5 * 2048 + 2 * E + E // 3 + 1
        x = special_values(dtype, n, bits * 29 + E)
        ref = oracle.compress(x, bits, E, canary=0x44)
        want = oracle.decompress(ref, n, dtype, bits, E)
        size = ref.size
        for voff in (0, 1):
            tv = torch.zeros(n + 4, dtype=tdt, device="cuda")
            tv[voff:voff + n] = torch.from_numpy(x).cuda()
            buf = torch.full((size,), 0x44, dtype=torch.uint8, device="cuda")
            frsz_b200.compress(tv[voff:voff + n], bits, E, out=buf)
            got = buf.cpu().numpy()
            if not np.array_equal(got, ref):
                bad = np.flatnonzero(got != ref)
                raise AssertionError(f"bits={bits} E={E} voff={voff}: {bad.size} bytes differ, first {bad[:6]}")
        for voff in (0, 1):
            out = torch.full((n + 4,), -7.0, dtype=tdt, device="cuda")
            frsz_b200.decompress(torch.from_numpy(ref).cuda(), n, dtype, bits, E, out=out[voff:voff + n])
            got = out.cpu().numpy()
            assert np.array_equal(got[voff:voff + n].view(uint), want.view(uint)), (bits, E, voff)
            assert np.all(got[:voff] == -7.0) and np.all(got[voff + n:] == -7.0), (bits, E, voff)


@pytest.mark.parametrize("E", [17, 19, 24, 48, 100, 127, 128 - 1])
def test_blocks_17_to_128_whole_chunks(cuda, E):
    """Arrays of exactly whole chunks (the chunked kernels take 2048 // E
    blocks at a time, so a chunk holds up to E - 1 values fewer than 2048):
    the last chunk is full and nothing is written past the array."""
    for dtype, bits in ((np.float32, 16), (np.float32, 5), (np.float64, 21), (np.float64, 40)):
        es = np.dtype(dtype).itemsize
        tdt = torch.float32 if es == 4 else torch.float64
        uint = np.uint32 if es == 4 else np.uint64
        n = (2048 // E) * E * 3
        x = special_values(dtype, n, bits + E)
        check(x, bits, E)
        ref = oracle.compress(x, bits, E, canary=0x44)
        out = torch.full((n + 256,), -7.0, dtype=tdt, device="cuda")
        frsz_b200.decompress(torch.from_numpy(ref).cuda(), n, dtype, bits, E, out=out[:n])
        got = out.cpu().numpy()
        assert np.array_equal(got[:n].view(uint), oracle.decompress(ref, n, dtype, bits, E).view(uint)), (bits, E)
        assert np.all(got[n:] == -7.0), (bits, E)
