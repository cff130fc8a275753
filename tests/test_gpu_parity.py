"""GPU parity: the sm_100a kernels, called through the C ABI, against the
oracle and the reference's golden fixtures.  Integer/byte work: bit-exact
(whole compressed buffers including canary bytes, decompressed values by bit
pattern)."""
import hashlib
import importlib.util
import json
import os

import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import workloads

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def gpu_compress(x: np.ndarray, bits: int, E: int, canary: int = 0xFF, slack: int = 0) -> np.ndarray:
    size = frsz_b200.compressed_size(x.dtype, bits, E, x.size)
    buf = torch.full((size + slack,), canary, dtype=torch.uint8, device="cuda")
    frsz_b200.compress(torch.from_numpy(np.ascontiguousarray(x)).cuda(), bits, E, out=buf)
    torch.cuda.synchronize()
    return buf.cpu().numpy()


def gpu_decompress(buf: np.ndarray, n: int, dtype, bits: int, E: int) -> np.ndarray:
    d = torch.from_numpy(np.ascontiguousarray(buf)).cuda()
    y = frsz_b200.decompress(d, n, dtype, bits, E)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def same_values(a: np.ndarray, b: np.ndarray) -> bool:
    return a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_reference_e2e_fixtures(cuda):
    """The reference GPU test's 11 end-to-end cases: the whole 0xFF-canary
    buffer (+128 slack) byte-identical to the reference CPU codec's, and a
    lossless decode (test/test_frsz_gpu.cu:316-410)."""
    g = np.load(os.path.join(GOLDEN, "e2e_reference_test.npz"))
    for key in g.files:
        dt, b, e = key.split("_")
        bits, E = int(b[1:]), int(e[1:])
        dtype = np.float64 if dt == "float64" else np.float32
        n = 2049 if dtype == np.float64 else 2160
        x = workloads.reference_pattern(n, dtype)
        buf = gpu_compress(x, bits, E, 0xFF, slack=128)
        assert np.array_equal(buf, g[key]), key
        assert same_values(gpu_decompress(buf, n, dtype, bits, E), x), key


def test_back_and_forth32(cuda):
    g = np.load(os.path.join(GOLDEN, "back_and_forth32.npz"))
    x = g["input"]
    buf = gpu_compress(x, 32, 1, 0xFF, slack=128)
    assert np.array_equal(buf, g["compressed"])
    assert same_values(gpu_decompress(buf, x.size, np.float32, 32, 1), x)


def test_digest_fixtures(cuda):
    """1080 seeded cases across every bits / block size / float type, against
    SHA-256 digests of the reference codec's output."""
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = json.load(open(os.path.join(GOLDEN, "digests.json")))
    bad = []
    for c in d["cases"]:
        dt = np.dtype(c["dtype"]).type
        x = mg.random_case_input(dt, c["bits"], c["E"], c["n"], c["seed"])
        comp = gpu_compress(x, c["bits"], c["E"], canary=0xA5)
        ok_c = _sha(comp) == c["compressed_sha256"]
        dec = gpu_decompress(comp if ok_c else oracle.compress(x, c["bits"], c["E"], canary=0xA5), c["n"], dt,
                             c["bits"], c["E"])
        ok_d = _sha(dec) == c["decompressed_sha256"]
        if not (ok_c and ok_d):
            bad.append((c["dtype"], c["bits"], c["E"], c["n"], ok_c, ok_d))
    assert not bad, f"{len(bad)} mismatches, first: {bad[:8]}"


def test_fp64_2p20_round_trip(cuda):
    """The CPU-parity round trip, fp64 2^20 N(0,1), E 32, 32 bits -- bytes and values equal the
    reference's (digests)."""
    c = json.load(open(os.path.join(GOLDEN, "digests.json")))["fp64_2p20_round_trip"]
    x = workloads.normal_np(c["n"], np.float64, c["seed"])
    comp = gpu_compress(x, 32, 32, canary=0xFF)
    assert _sha(comp) == c["compressed_sha256"]
    assert _sha(gpu_decompress(comp, c["n"], np.float64, 32, 32)) == c["decompressed_sha256"]


@pytest.mark.parametrize("dtype,bits,E,n", [
    (np.float32, 16, 32, 4096 * 37 + 1),
    (np.float32, 8, 32, 4096 * 11),
    (np.float32, 12, 32, 300_001),
    (np.float32, 24, 32, 123_457),
    (np.float32, 32, 32, 99_999),
    (np.float32, 5, 64, 50_000),
    (np.float32, 13, 8, 40_000),
    (np.float32, 16, 1024, 70_000),
    (np.float32, 31, 4096, 9_000),
    (np.float64, 16, 32, 2048 * 40 + 7),
    (np.float64, 21, 32, 500_001),
    (np.float64, 32, 32, 250_000),
    (np.float64, 16, 64, 131_072),
    (np.float64, 21, 64, 131_075),
    (np.float64, 32, 64, 77_777),
    (np.float64, 8, 32, 60_000),
    (np.float64, 12, 32, 60_003),
    (np.float64, 24, 32, 60_001),
    (np.float64, 33, 32, 40_000),
    (np.float64, 47, 16, 40_001),
    (np.float64, 64, 32, 40_000),
    (np.float64, 63, 128, 33_333),
    (np.float64, 40, 1024, 20_000),
    (np.float64, 52, 2048, 10_000),
])
def test_random_vs_oracle(cuda, dtype, bits, E, n):
    lo, hi = (-30, 30) if (dtype == np.float64 and bits <= 8) else ((-300, 300) if dtype == np.float64 else (-35, 35))
    x = workloads.loguniform_np(n, dtype, seed=bits * 1000 + E, lo=lo, hi=hi)
    ref = oracle.compress(x, bits, E, canary=0x5A, threads=4)
    got = gpu_compress(x, bits, E, canary=0x5A)
    assert np.array_equal(got, ref)
    y = gpu_decompress(ref, n, dtype, bits, E)
    assert same_values(y, oracle.decompress(ref, n, dtype, bits, E, threads=4))


@pytest.mark.parametrize("dtype,bits,E", [(np.float32, 16, 32), (np.float64, 21, 32), (np.float64, 64, 8)])
def test_unaligned_pointers_use_generic_path(cuda, dtype, bits, E):
    """Value and buffer pointers that are only element/word aligned."""
    n = 10_001
    x = workloads.normal_np(n, dtype, 3)
    es = np.dtype(dtype).itemsize
    w = frsz_b200.word_bits(bits) // 8
    size = frsz_b200.compressed_size(dtype, bits, E, n)
    tv = torch.zeros(n + 1, dtype=torch.float32 if dtype == np.float32 else torch.float64, device="cuda")
    tv[1:] = torch.from_numpy(x).cuda()
    raw = torch.full((size + 64,), 0x77, dtype=torch.uint8, device="cuda")
    off = w if w < 16 else 8
    if frsz_b200.word_bits(bits) == 64:
        off = 8
    buf = raw[off:off + size]
    frsz_b200.compress(tv[1:], bits, E, out=buf)
    torch.cuda.synchronize()
    ref = oracle.compress(x, bits, E, canary=0x77)
    assert np.array_equal(buf.cpu().numpy(), ref)
    y = torch.zeros_like(tv)
    frsz_b200.decompress(buf, n, dtype, bits, E, out=y[1:])
    torch.cuda.synchronize()
    assert same_values(y[1:].cpu().numpy(), oracle.decompress(ref, n, dtype, bits, E))
    assert es in (4, 8)


@pytest.mark.parametrize("dtype,bits,E", [(np.float32, 16, 32), (np.float64, 21, 32), (np.float64, 64, 5),
                                          (np.float32, 9, 5)])
def test_random_access_elements(cuda, dtype, bits, E):
    n = 20_000
    x = workloads.loguniform_np(n, dtype, 4, lo=-20, hi=20)
    comp = oracle.compress(x, bits, E)
    idx = np.random.default_rng(1).integers(0, n, 3000)
    got = frsz_b200.decompress_elements(torch.from_numpy(comp).cuda(), n, dtype, bits, E,
                                        torch.from_numpy(idx).cuda()).cpu().numpy()
    want = np.array([oracle.decompress_element(comp, n, dtype, bits, E, int(i)) for i in idx], dtype=dtype)
    assert same_values(got, want)


@pytest.mark.parametrize("dtype,bits,E,n", [(np.float32, 16, 32, 1_000_003), (np.float64, 21, 32, 700_001),
                                            (np.float64, 9, 5, 100_000),
                                            # several 64 MiB pipeline slices, ragged tail
                                            (np.float32, 12, 32, 40_000_123), (np.float64, 21, 64, 20_000_077),
                                            (np.float64, 13, 5, 9_000_011)])
def test_host_buffers(cuda, dtype, bits, E, n):
    """frsz2_compress_host / frsz2_decompress_host: bytes the reference never
    writes keep the caller's canary."""
    x = workloads.loguniform_np(n, dtype, 8, lo=-25, hi=25)
    out = np.full(frsz_b200.compressed_size(dtype, bits, E, n), 0xC3, dtype=np.uint8)
    pinned = torch.from_numpy(x).pin_memory().numpy()
    frsz_b200.compress_host(pinned, bits, E, out=out)
    ref = oracle.compress(x, bits, E, canary=0xC3, threads=4)
    assert np.array_equal(out, ref)
    y = frsz_b200.decompress_host(out, n, dtype, bits, E)
    assert same_values(y, oracle.decompress(ref, n, dtype, bits, E, threads=4))


def test_empty_and_tiny(cuda):
    for dtype in (np.float32, np.float64):
        for n in (0, 1, 2, 7):
            x = workloads.normal_np(n, dtype, 1)
            for bits, E in ((16, 32), (8, 1), (32, 8)):
                assert np.array_equal(gpu_compress(x, bits, E, 0x11), oracle.compress(x, bits, E, 0x11))


def test_compressor_view_and_dispatch(cuda):
    """The reference-shaped API: Frsz2Compressor views and runtime dispatch."""
    n = 10_000
    x = torch.from_numpy(workloads.normal_np(n, np.float64, 2)).cuda()
    buf = torch.full((frsz_b200.compressed_size(np.float64, 16, 64, n),), 0xFF, dtype=torch.uint8, device="cuda")
    frsz_b200.dispatch_frsz2_compression(np.float64, range(4, 65), 16, [2, 4, 8, 16, 32, 64], 64, x, n, buf)
    y = torch.empty_like(x)
    frsz_b200.dispatch_frsz2_decompression(np.float64, range(4, 65), 16, [2, 4, 8, 16, 32, 64], 64, y, n, buf)
    torch.cuda.synchronize()
    ref = oracle.compress(x.cpu().numpy(), 16, 64, 0xFF)
    assert np.array_equal(buf.cpu().numpy(), ref)
    assert same_values(y.cpu().numpy(), oracle.decompress(ref, n, np.float64, 16, 64))
    view = frsz_b200.Frsz2Compressor(16, 64, np.float64, buf, n)
    assert torch.equal(view.get_exponent_data().cpu(),
                       torch.from_numpy(ref[: view.get_exponent_data().numel() * 2].view(np.int16).copy()))


@pytest.mark.parametrize("dtype,bits,E", [(np.float32, 16, 32), (np.float32, 9, 5), (np.float32, 21, 8),
                                          (np.float64, 21, 32), (np.float64, 33, 32), (np.float64, 7, 1),
                                          (np.float64, 64, 1000)])
def test_host_random_access_matches_oracle(cuda, dtype, bits, E):
    """frsz2_decompress_elements_host: host buffer, host indices (duplicates,
    any order, some out of range), host outputs."""
    rng = np.random.default_rng(bits * 7 + E)
    n = 10_007
    lo, hi = (-30, 30) if dtype == np.float64 and bits <= 8 else (-20, 20)
    x = workloads.loguniform_np(n, dtype, seed=bits + E, lo=lo, hi=hi)
    x[rng.choice(n, 50, replace=False)] = 0.0
    x[rng.choice(n, 20, replace=False)] = np.nan
    ref = oracle.compress(x, bits, E)
    want = oracle.decompress(ref, n, dtype, bits, E)
    idx = np.concatenate([rng.integers(0, n, 3000), [0, n - 1, n - 1, 5, n, n + 77, 2 ** 63]]).astype(np.uint64)
    out = np.full(idx.size, 42.0, dtype=dtype)
    frsz_b200.decompress_elements_host(ref, n, dtype, bits, E, idx, out=out)
    valid = idx < n
    uint = np.uint64 if dtype == np.float64 else np.uint32
    assert np.array_equal(out[valid].view(uint), want[idx[valid].astype(np.int64)].view(uint))
    assert np.all(out[~valid] == 42.0)
