"""CPU: the oracle restatement pinned against the reference's known answers,
its golden fixtures, and (where built) the reference library itself."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from frsz_b200 import workloads

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
L = oracle.oracle_lib()


def f32(bits):
    return np.array([bits], dtype=np.uint32).view(np.float32)[0]


def f64(bits):
    return np.array([bits], dtype=np.uint64).view(np.float64)[0]


# ---------------------------------------------------------------- known answers

def test_bit_cast_known_answers():
    """test/test_frsz_gpu.cu:88-158: bit patterns of special values."""
    ui32 = [0b0_01111111_01000000000000000000000, 0b0_00000000_00000000000000000000001,
            0b0_00000001_00000000000000000000000, 0b1_11111111_00000000000000000000000, 0,
            0b1_01111111_00000000000000000000001, 0b0_01101000_00000000000000000000000,
            0b0_10000011_01010000000000000000000]
    e32 = np.finfo(np.float32).eps
    fl32 = [1.25, np.finfo(np.float32).smallest_subnormal, np.finfo(np.float32).tiny, -np.inf, 0.0,
            -1 - e32, e32, 21.0]
    assert np.array_equal(np.array(ui32, dtype=np.uint32).view(np.float32), np.array(fl32, dtype=np.float32))
    ui64 = [0b0_01111111111 << 52 | 1 << 50, 1, 1 << 52, 0b1_11111111111 << 52, 0, (0b1_01111111111 << 52) | 1,
            0b0_01111001011 << 52, (0b0_10000000011 << 52) | (0b0101 << 48)]
    e64 = np.finfo(np.float64).eps
    fl64 = [1.25, np.finfo(np.float64).smallest_subnormal, np.finfo(np.float64).tiny, -np.inf, 0.0,
            -1 - e64, e64, 21.0]
    assert np.array_equal(np.array(ui64, dtype=np.uint64).view(np.float64), np.array(fl64, dtype=np.float64))


def test_dismantling_known_answers():
    """test/test_frsz_gpu.cu:213-229."""
    for x, s, e, m in zip([32.0, 0.5, 0.0, -0.375], [0, 0, 0, 1], [5, -1, -127, -2],
                          [1 << 23, 1 << 23, 0, 3 << 22]):
        assert L.frsz2o_sign_f32(x) == s
        assert L.frsz2o_exponent_f32(x) == e
        assert L.frsz2o_significand_f32(x) == m
    for x, s, e, m in zip([-32.0, 0.5, 0.0, -0.375], [1, 0, 0, 1], [5, -1, -1023, -2],
                          [1 << 52, 1 << 52, 0, 3 << 51]):
        assert L.frsz2o_sign_f64(x) == s
        assert L.frsz2o_exponent_f64(x) == e
        assert L.frsz2o_significand_f64(x) == m


def test_floating_to_fixed_known_answers():
    """test/test_frsz_gpu.cu:276-301, including the zero/subnormal rule: a
    subnormal at block exponent 5 truncates to 0 and decodes to 2^(5-31)."""
    in32 = [32.0, 2.0, f32(0b0_00000000_11111111111111111111111), 0.125, -0.375]
    exp32 = [5, 5, 5, 2, 1]
    mid32 = [0x800000 << 7, 0x800000 << 3, 0, 0x02000000, 0x8C000000]
    out32 = [32.0, 2.0, f32(0b0_01100101_00000000000000000000000), 0.125, -0.375]
    for x, e, mid, y in zip(in32, exp32, mid32, out32):
        r = L.frsz2o_floating_to_fixed_f32(x, e)
        assert r == mid
        assert np.float32(L.frsz2o_fixed_to_floating_f32(r, e)).view(np.uint32) == np.float32(y).view(np.uint32)
    in64 = [32.0, 2.0, -0.125, 0.375]
    exp64 = [5, 5, 2, -1]
    mid64 = [1 << 62, 1 << 58, 0x82 << 56, 3 << 60]
    for x, e, mid in zip(in64, exp64, mid64):
        r = L.frsz2o_floating_to_fixed_f64(x, e)
        assert r == mid
        assert L.frsz2o_fixed_to_floating_f64(r, e) == x
    # test/test_frsz.cc:561-563 (restated helpers, same rule)
    sub = f32(0b0000000001111111111111111111111)
    assert np.float32(L.frsz2o_fixed_to_floating_f32(L.frsz2o_floating_to_fixed_f32(sub, 5), 5)).view(
        np.uint32) == 0b00110010100000000000000000000000


def test_zero_code_quirk_fp64():
    """clz of a zero 64-bit magnitude counts 32 (frsz2.hpp:180-186): zero
    codes decode to 2^(e_b-31) in fp64 too, and to 0 when e_b+bias < 31."""
    assert L.frsz2o_fixed_to_floating_f64(0, 3) == 2.0 ** (3 - 31)
    assert L.frsz2o_fixed_to_floating_f64(1 << 63, 3) == -(2.0 ** (3 - 31))
    assert L.frsz2o_fixed_to_floating_f64(0, -1023) == 0.0
    assert L.frsz2o_fixed_to_floating_f32(0, 3) == np.float32(2.0 ** (3 - 31))


# ---------------------------------------------------------------- size algebra

@pytest.mark.parametrize("bits,E,n,expect", [
    (32, 32, 1 << 20, 4325632),       # fp64 2^20, E 32, 32 bits: 32768*4 + 256 pad + 32768*128
    (16, 32, 512 ** 3, 8388608 + 256 + (1 << 22) * 64),
    (21, 32, 1 << 28, (1 << 23) * 4 + 256 + (1 << 23) * 84),
    (32, 32, 0, 256),                 # empty: a full pad
    (8, 32, 256, 8 + 248 + 8 * 32),   # exponent array not aligned: pad to 256
    (8, 1, 256, 256 + 256 + 256),     # already aligned: a full extra 256 B
])
def test_sizes(bits, E, n, expect):
    assert oracle.compressed_bytes(bits, E, n) == expect


# ---------------------------------------------------------------- golden fixtures

def test_reference_e2e_fixtures():
    """The reference GPU test's end-to-end cases: whole canary buffer equal to
    what the reference wrote, and a lossless round trip (test_frsz_gpu.cu:347-376)."""
    g = np.load(os.path.join(GOLDEN, "e2e_reference_test.npz"))
    assert len(g.files) == 11
    for key in g.files:
        dt, b, e = key.split("_")
        bits, E = int(b[1:]), int(e[1:])
        dtype = np.float64 if dt == "float64" else np.float32
        n = 2049 if dtype == np.float64 else 2160
        x = workloads.reference_pattern(n, dtype)
        buf = np.full(oracle.compressed_bytes(bits, E, n) + 128, 0xFF, dtype=np.uint8)
        rc = getattr(L, f"frsz2o_compress_{'f64' if dtype == np.float64 else 'f32'}")(
            x.ctypes.data, n, bits, E, buf.ctypes.data)
        assert rc == 0
        assert np.array_equal(buf, g[key]), key
        y = oracle.decompress(buf, n, dtype, bits, E)
        assert np.array_equal(y, x), key


def test_back_and_forth32_fixture():
    g = np.load(os.path.join(GOLDEN, "back_and_forth32.npz"))
    x = g["input"]
    buf = np.full(oracle.compressed_bytes(32, 1, x.size) + 128, 0xFF, dtype=np.uint8)
    L.frsz2o_compress_f32(x.ctypes.data, x.size, 32, 1, buf.ctypes.data)
    assert np.array_equal(buf, g["compressed"])
    assert np.array_equal(oracle.decompress(buf, x.size, np.float32, 32, 1), x)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def test_digest_fixtures():
    """1080 seeded cases over every bits / block size / float type: the
    oracle reproduces the reference's bytes and values (SHA-256)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = json.load(open(os.path.join(GOLDEN, "digests.json")))
    bad = []
    for c in d["cases"]:
        dt = np.dtype(c["dtype"]).type
        x = mg.random_case_input(dt, c["bits"], c["E"], c["n"], c["seed"])
        comp = oracle.compress(x, c["bits"], c["E"], canary=0xA5)
        dec = oracle.decompress(comp, c["n"], dt, c["bits"], c["E"])
        if _sha(comp) != c["compressed_sha256"] or _sha(dec) != c["decompressed_sha256"]:
            bad.append((c["dtype"], c["bits"], c["E"], c["n"]))
    assert not bad, bad[:10]
    c = d["fp64_2p20_round_trip"]
    x = workloads.normal_np(c["n"], np.float64, c["seed"])
    comp = oracle.compress(x, 32, 32, canary=0xFF)
    assert _sha(comp) == c["compressed_sha256"]
    assert _sha(oracle.decompress(comp, c["n"], np.float64, 32, 32)) == c["decompressed_sha256"]


def test_threaded_oracle_matches_serial():
    x = workloads.loguniform_np(100_003, np.float64, 5, lo=-20, hi=20)
    a = oracle.compress(x, 21, 32)
    b = oracle.compress(x, 21, 32, threads=4)
    assert np.array_equal(a, b)
    assert np.array_equal(oracle.decompress(a, x.size, np.float64, 21, 32),
                          oracle.decompress(a, x.size, np.float64, 21, 32, threads=3))


def test_error_bound_holds():
    """|x - x_hat| <= per-block bound 2^(e_b - bits + 2) (truncation twice)."""
    x = workloads.loguniform_np(1 << 14, np.float64, 9, lo=-10, hi=10)
    for bits in (16, 21, 32):
        comp = oracle.compress(x, bits, 32)
        y = oracle.decompress(comp, x.size, np.float64, bits, 32)
        nb = -(-x.size // 32)
        be = comp[: nb * 4].view(np.int32) if bits > 16 else comp[: nb * 2].view(np.int16)
        bound = np.repeat(oracle.error_bound(be, bits), 32)[: x.size]
        assert np.all(np.abs(x - y) <= bound)


# ---------------------------------------------------------------- reference library

@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_oracle_matches_reference_random():
    rng = np.random.default_rng(3)
    for _ in range(300):
        dtype = np.float64 if rng.random() < 0.5 else np.float32
        bits = int(rng.integers(4, 65 if dtype == np.float64 else 33))
        E = int(rng.choice([1, 2, 4, 5, 8, 16, 32, 64, 128, 256, 512, 1024]))
        n = int(rng.integers(0, 3000))
        x = workloads.loguniform_np(n, dtype, int(rng.integers(1 << 30)),
                                    lo=-30 if (dtype == np.float64 and bits <= 8) else -35,
                                    hi=30 if dtype == np.float64 else 35)
        a = oracle.compress(x, bits, E, canary=0x3C)
        b = oracle.ref_compress(x, bits, E, canary=0x3C)
        assert np.array_equal(a, b), (dtype, bits, E, n)
        ya = oracle.decompress(a, n, dtype, bits, E)
        yb = oracle.ref_decompress(b, n, dtype, bits, E)
        assert np.array_equal(ya.view(np.uint8), yb.view(np.uint8)), (dtype, bits, E, n)
        if n:
            i = int(rng.integers(n))
            ea = oracle.decompress_element(a, n, dtype, bits, E, i)
            eb = (oracle.ref_lib().frsz2ref_decompress_element_f64 if dtype == np.float64
                  else oracle.ref_lib().frsz2ref_decompress_element_f32)(bits, E, b.ctypes.data, n, i)
            assert np.array([ea], dtype=dtype).view(np.uint8).tobytes() == \
                np.array([eb], dtype=dtype).view(np.uint8).tobytes()


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_oracle_primitives_match_reference():
    R = oracle.ref_lib()
    rng = np.random.default_rng(11)
    xs32 = np.concatenate([rng.standard_normal(200).astype(np.float32),
                           np.array([0, -0.0, 1e-42, -3e-39, 3.4e38], dtype=np.float32)])
    for x in xs32:
        x = float(x)
        assert L.frsz2o_exponent_f32(x) == R.frsz2ref_exponent_f32(x)
        assert L.frsz2o_significand_f32(x) == R.frsz2ref_significand_f32(x)
        for e in (-127, -20, 0, 3, 127):
            if e >= L.frsz2o_exponent_f32(x):
                r = L.frsz2o_floating_to_fixed_f32(x, e)
                assert r == R.frsz2ref_floating_to_fixed_f32(x, e)
                assert np.float32(L.frsz2o_fixed_to_floating_f32(r, e)).view(np.uint32) == \
                    np.float32(R.frsz2ref_fixed_to_floating_f32(r, e)).view(np.uint32)
    for x in np.concatenate([rng.standard_normal(200), [0.0, 5e-320, -2e-310, 1e300]]):
        x = float(x)
        assert L.frsz2o_exponent_f64(x) == R.frsz2ref_exponent_f64(x)
        assert L.frsz2o_significand_f64(x) == R.frsz2ref_significand_f64(x)
        for e in (-1023, -100, 0, 5, 1023):
            if e >= L.frsz2o_exponent_f64(x):
                r = L.frsz2o_floating_to_fixed_f64(x, e)
                assert r == R.frsz2ref_floating_to_fixed_f64(x, e)
                assert L.frsz2o_fixed_to_floating_f64(r, e) == R.frsz2ref_fixed_to_floating_f64(r, e)


# ---------------------------------------------------------------- property-based

from hypothesis import HealthCheck, given, settings, strategies as st  # noqa: E402


def _finite_or_nan(dtype, allow_nan):
    return st.floats(allow_nan=allow_nan, allow_infinity=False, allow_subnormal=True, width=32 if dtype == np.float32 else 64)


@st.composite
def codec_case(draw):
    is64 = draw(st.booleans())
    dtype = np.float64 if is64 else np.float32
    bits = draw(st.integers(4, 64 if is64 else 32))
    E = draw(st.sampled_from([1, 2, 4, 5, 8, 16, 32, 64, 128]))
    n = draw(st.integers(0, 400))
    # NaN is defined in the reference for fp32 blocks (std::max skips it and the
    # shift stays below the word width); fp64 NaN elements shift past the word
    vals = draw(st.lists(_finite_or_nan(dtype, allow_nan=not is64), min_size=n, max_size=n))
    x = np.array(vals, dtype=dtype)
    if is64 and bits <= 8:
        x = np.clip(x, -1e38, 1e38)  # |x| >= 2^128 wraps the int8 exponent into undefined shifts
    return x, bits, E


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@settings(max_examples=300, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(codec_case())
def test_property_oracle_equals_reference(case):
    x, bits, E = case
    a = oracle.compress(x, bits, E, canary=0x96)
    b = oracle.ref_compress(x, bits, E, canary=0x96)
    assert np.array_equal(a, b)
    ya = oracle.decompress(a, x.size, x.dtype, bits, E)
    yb = oracle.ref_decompress(b, x.size, x.dtype, bits, E)
    assert np.array_equal(ya.view(np.uint8), yb.view(np.uint8))
