"""The legacy "frsz" codec (src/frsz.cc:15-165): the oracle against the
reference test's known answer (test/test_frsz.cc:29-46) on CPU, and the CUDA
kernels against the oracle, bit for bit, on the GPU -- int16 streams and
decoded values, in both decode modes (the reference's use of block 0's
differences, and each block's own)."""
import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import legacy, workloads


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_reference_known_answer(dtype):
    # test/test_frsz.cc:29-46: epsilon 5, {10, 20, 30, 20, 10} round trips
    x = np.array([10.0, 20.0, 30.0, 20.0, 10.0], dtype=dtype)
    q = oracle.frsz1_compress(x, 5.0)
    assert q.tolist() == [1, 1, 1, -1, -1]
    assert np.array_equal(oracle.frsz1_decompress(q, dtype, 5.0), x)


def test_oracle_block_rules():
    # differences restart every 256 values; saturation at the int16 limits;
    # the reference decoder adds block 0's differences in later blocks
    x = np.arange(600, dtype=np.float64) * 2.0
    q = oracle.frsz1_compress(x, 0.5)  # step 1: quantized values 0, 2, 4, ...
    assert q[0] == 0 and q[256] == 512 and q[512] == 1024 and np.all(q[1:256] == 2)
    # differences: 5e8, -1e9, +Inf (Inf - -5e8), NaN (NaN - Inf)
    big = oracle.frsz1_compress(np.array([1e9, -1e9, np.inf, np.nan], dtype=np.float32), 1.0)
    assert big.tolist() == [32767, -32768, 32767, 0]
    y_ref = oracle.frsz1_decompress(q, np.float64, 0.5)
    y_own = oracle.frsz1_decompress(q, np.float64, 0.5, own_deltas=True)
    assert np.array_equal(y_own, x)
    assert np.array_equal(y_ref[:256], x[:256])
    # block 1 starts from its own first value, then adds block 0's differences
    assert y_ref[256] == x[256] and y_ref[257] == x[256] + 2.0


# ------------------------------------------------------------------ known answers
# Each case below is worked out by hand from the reference's lines: the
# quantizer quantized[i] = std::round(data[i] * ebx2_inv) (src/frsz.cc:125,
# half away from zero, in double), the difference within blocks of 256
# (:128-129) and saturate<int16_t> (:99-103); the decoder's per-block loop
# `for block_idx < (len/BLOCK)+1` with `if (BLOCK*block_idx < len)` and its
# running sum over quantized[i], i the index within the block (:140-151).

HALF = np.nextafter(0.5, 0.0)  # 0.49999999999999994


def fp32_eps_for(p_target: float, seed_x: float):
    """A float x and an epsilon for which (double) x * (1 / (2 eps)) is
    exactly p_target: searched over floats x near seed_x and, for each, the
    doubles next to x / (2 p_target)."""
    xf = np.float32(seed_x)
    for _ in range(64):
        e0 = float(xf) / (2.0 * p_target)
        for d in range(-64, 65):
            e = e0
            step = np.inf if d > 0 else -np.inf
            for _ in range(abs(d)):
                e = np.nextafter(e, step)
            if float(xf) * (1.0 / (e * 2.0)) == p_target:
                return xf, float(e)
        xf = np.nextafter(xf, np.float32(np.inf))
    raise AssertionError(f"no float and epsilon give {p_target!r}")


def rounding_known_answers():
    """(dtype, x, epsilon, expected int16 stream)."""
    out = [
        # epsilon 0.5: step 1, p = x.  Ties go away from zero (2.5 -> 3, not 2);
        # the double below 0.5 rounds to 0; one ulp either side of 2.5 gives 2
        # and 3; -HALF gives -0.  Differences: 1-0, 2-1, 3-2, -1-3, -3+1, 0+3,
        # 2-0, 3-2, -0-3.
        (np.float64, [0.5, 1.5, 2.5, -0.5, -2.5, HALF, np.nextafter(2.5, 0), np.nextafter(2.5, 9), -HALF], 0.5,
         [1, 1, 1, -4, -2, 3, 2, 1, -3]),
        # a float input whose p is the double just below 0.5: q = 0
        (np.float32, [3.202960252761841], 3.2029602527618413, [0]),
    ]
    # float inputs with p one double-ulp either side of k + 0.5: q = k, then k + 1
    for k in (0, 1, 2, 7, 100, 4095):
        xl, lo = fp32_eps_for(np.nextafter(k + 0.5, 0.0), 2 * k + 1.37)
        xh, hi = fp32_eps_for(np.nextafter(k + 0.5, np.inf), 2 * k + 1.37)
        out.append((np.float32, [xl], lo, [k]))
        out.append((np.float32, [xh], hi, [k + 1]))
        out.append((np.float32, [-xh], hi, [-(k + 1)]))
    return out


def saturation_known_answers():
    return [
        # epsilon 0.5: q = x.  Differences 32767, 32768 (-> 32767), -32768
        # (exact, not saturated), -32768, 40001 (-> 32767), -80000 (-> -32768),
        # 40000 (-> 32767)
        (np.float64, [32767, 65535, 32767, -1, 40000, -40000, 0], 0.5,
         [32767, 32767, -32768, -32768, 32767, -32768, 32767]),
        (np.float32, [32767, 65535, 32767, -1, 40000, -40000, 0], 0.5,
         [32767, 32767, -32768, -32768, 32767, -32768, 32767]),
        # +-Inf: differences +Inf, -Inf, +Inf, Inf - Inf = NaN (0, the value
        # x86 code gives the undefined conversion), -Inf, +Inf
        (np.float32, [np.inf, 0, np.inf, np.inf, -np.inf, 5], 0.5, [32767, -32768, 32767, 0, -32768, 32767]),
        (np.float64, [np.inf, 0, np.inf, np.inf, -np.inf, 5], 0.5, [32767, -32768, 32767, 0, -32768, 32767]),
    ]


def block_restart_known_answer():
    # the difference restarts at i = 256: 30000 - 0, not 30000 - 30000
    x = np.full(258, 30000.0)
    want = np.zeros(258, dtype=np.int16)
    want[0] = want[256] = 30000
    return x, want


def decode_streams():
    """(n, int16 stream, expected values with the reference's decode, with
    each block's own differences); epsilon 0.5, so 2 eps = 1.  Block 0 holds
    [0, 1, 1, ...]; block 1 starts at 100 and holds 2s; block 2 starts at -7
    and holds 5s.  The reference adds block 0's differences (1) in every
    block: block 1 decodes as 100 + i, block 2 as -7 + i; its own 2s and 5s
    give 100 + 2i and -7 + 5i.  n = 512 is a multiple of 256, where the
    (len/BLOCK)+1-th block is empty; n = 257 leaves block 1 one value."""
    out = []
    for n in (257, 512, 600):
        q = np.ones(n, dtype=np.int16)
        q[0] = 0
        q[256:512] = 2
        q[256] = 100
        if n > 512:
            q[512:] = 5
            q[512] = -7
        ref = np.empty(n)
        own = np.empty(n)
        for i in range(n):
            b, j = divmod(i, 256)
            ref[i] = j if b == 0 else (100 + j if b == 1 else -7 + j)
            own[i] = j if b == 0 else (100 + 2 * j if b == 1 else -7 + 5 * j)
        out.append((n, q, ref, own))
    return out


@pytest.mark.parametrize("dtype,x,eps,want", rounding_known_answers() + saturation_known_answers())
def test_oracle_quantizer_known_answers(dtype, x, eps, want):
    with np.errstate(invalid="ignore"):
        got = oracle.frsz1_compress(np.array(x, dtype=dtype), eps)
    assert got.tolist() == want


def test_oracle_block_restart_and_decode_known_answers():
    x, want = block_restart_known_answer()
    for dtype in (np.float32, np.float64):
        assert np.array_equal(oracle.frsz1_compress(x.astype(dtype), 0.5), want)
    for n, q, ref, own in decode_streams():
        for dtype in (np.float32, np.float64):
            assert np.array_equal(oracle.frsz1_decompress(q, dtype, 0.5), ref.astype(dtype)), n
            assert np.array_equal(oracle.frsz1_decompress(q, dtype, 0.5, own_deltas=True), own.astype(dtype)), n


@pytest.mark.gpu
def test_gpu_known_answers(cuda):
    """The kernels give the hand-derived answers above, bit for bit; decoding
    writes nothing past n (canary slack)."""
    for dtype, x, eps, want in rounding_known_answers() + saturation_known_answers():
        t = torch.from_numpy(np.array(x, dtype=dtype)).cuda()
        assert legacy.compress(t, eps).cpu().tolist() == want, (dtype, x, eps)
    x, want = block_restart_known_answer()
    for dtype in (np.float32, np.float64):
        assert np.array_equal(legacy.compress(torch.from_numpy(x.astype(dtype)).cuda(), 0.5).cpu().numpy(), want)
    for n, q, ref, own in decode_streams():
        for dtype, tdt in ((np.float32, torch.float32), (np.float64, torch.float64)):
            for own_deltas, expect in ((False, ref), (True, own)):
                out = torch.full((n + 64,), -3.0, dtype=tdt, device="cuda")
                legacy.decompress(torch.from_numpy(q).cuda(), tdt, 0.5, own_deltas=own_deltas, out=out[:n])
                got = out.cpu().numpy()
                assert np.array_equal(got[:n], expect.astype(dtype)), (n, dtype, own_deltas)
                assert np.all(got[n:] == -3.0), (n, dtype, own_deltas)


def test_plugin_surface():
    # src/frsz.cc:19-46, 82-86, 160; CMakeLists.txt:3 (project version)
    p = legacy.Frsz1Plugin()
    assert p.get_options() == {"frsz:epsilon": 1e-4}
    p.set_options({"frsz:epsilon": 0.25})
    assert p.epsilon == 0.25 and p.clone().get_options() == {"frsz:epsilon": 0.25}
    assert p.get_configuration() == {"pressio:thread_safe": "multiple", "pressio:stability": "experimental"}
    doc = p.get_documentation()
    assert doc["pressio:description"] == "a fixed rate version of the SZ Algorithm"
    assert doc["frsz:epsilon"].startswith('"absolute error bound" applied during quantization')
    assert (p.prefix, p.version(), p.major_version(), p.minor_version(), p.patch_version()) == ("frsz", "0.0.6", 0, 0, 6)
    assert p.get_metrics_results() == {}
    msg = "unsupported type: currently only floating point supported"
    assert p.compress(np.zeros(4, dtype=np.int32)) == (1, None) and (p.error_code, p.error_msg) == (1, msg)
    assert p.decompress(np.zeros(8, dtype=np.uint8), np.zeros(4, dtype=np.float16)) == 1


def test_plugin_length_rule():
    # normalized_dims(1).at(0) (src/frsz.cc:108, 139): unit extents dropped,
    # the first one left is the length, 0 when none is left
    assert legacy.legacy_length((1000,)) == 1000
    assert legacy.legacy_length((40, 54)) == 40
    assert legacy.legacy_length((1, 1, 7, 3)) == 7
    assert legacy.legacy_length((1,)) == 0 and legacy.legacy_length(()) == 0
    p = legacy.Frsz1Plugin()
    # nothing to code: no device work, an empty stream, the output untouched
    rc, buf = p.compress(np.ones((1, 1), dtype=np.float32))
    assert rc == 0 and buf.size == 0
    y = np.full(1, 7.0)
    assert p.decompress(buf, y) == 0 and y[0] == 7.0
    assert p.decompress(np.zeros(3, dtype=np.uint8), np.zeros(2)) == 2
    assert p.error_msg == "compressed input is shorter than the format requires"


def cases():
    rng = np.random.default_rng(5)
    out = []
    for dtype in (np.float32, np.float64):
        for n in (1, 7, 255, 256, 257, 1000, 65_536 + 13, (1 << 20) + 5):
            for eps in (1e-4, 0.5, 1e-7):
                x = workloads.normal_np(n, dtype, seed=n % 97) * dtype(10.0)
                if n > 10:
                    k = max(1, n // 200)
                    idx = rng.integers(0, n, (5, k))
                    x[idx[0]] = np.nan
                    x[idx[1]] = np.inf
                    x[idx[2]] = -np.inf
                    x[idx[3]] = -0.0
                    x[idx[4]] = dtype(3e8)
                out.append((x, eps))
    return out


@pytest.mark.gpu
def test_gpu_equals_oracle(cuda):
    for x, eps in cases():
        t = torch.from_numpy(x).cuda()
        q = legacy.compress(t, eps)
        want = oracle.frsz1_compress(x, eps)
        assert np.array_equal(q.cpu().numpy(), want), (x.dtype, x.size, eps)
        uint = np.uint64 if x.dtype == np.float64 else np.uint32
        for own in (False, True):
            y = legacy.decompress(torch.from_numpy(want).cuda(), t.dtype, eps, own_deltas=own).cpu().numpy()
            yw = oracle.frsz1_decompress(want, x.dtype, eps, own_deltas=own)
            assert np.array_equal(y.view(uint), yw.view(uint)), (x.dtype, x.size, eps, own)


@pytest.mark.gpu
def test_gpu_reference_known_answer_and_errors(cuda):
    x = torch.tensor([10.0, 20.0, 30.0, 20.0, 10.0], device="cuda")
    q = legacy.compress(x, 5.0)
    assert q.cpu().tolist() == [1, 1, 1, -1, -1]
    assert torch.equal(legacy.decompress(q, torch.float32, 5.0), x)
    lib = frsz_b200.lib()
    assert lib.frsz1_compressed_size(1000) == 2000
    assert lib.frsz1_compress(7, 1.0, x.data_ptr(), 5, q.data_ptr(), None) == frsz_b200.FRSZ2_EDTYPE
    assert b"only floating point" in lib.frsz2_last_error()
    assert lib.frsz1_compress(0, 0.0, x.data_ptr(), 5, q.data_ptr(), None) == frsz_b200.FRSZ2_EFAIL


@pytest.mark.gpu
def test_gpu_pointers_off_vector_alignment(cuda):
    n = 10_003
    x = workloads.normal_np(n, np.float32, seed=3)
    base = torch.zeros(n + 3, dtype=torch.float32, device="cuda")
    base[1:1 + n] = torch.from_numpy(x).cuda()
    out = torch.zeros(n + 3, dtype=torch.int16, device="cuda")
    q = legacy.compress(base[1:1 + n], 0.01, out=out[1:1 + n])
    assert np.array_equal(q.cpu().numpy(), oracle.frsz1_compress(x, 0.01))


@pytest.mark.gpu
def test_gpu_plugin_equals_oracle(cuda):
    # the plugin front end on host arrays and on device tensors: the same
    # int16 stream as the oracle (as bytes) and the reference decode
    p = legacy.Frsz1Plugin()
    p.set_options({"frsz:epsilon": 5.0})
    f = np.array([10.0, 20.0, 30.0, 20.0, 10.0], dtype=np.float32)  # test/test_frsz.cc:29-46
    rc, buf = p.compress(f)
    assert rc == 0 and buf.dtype == np.uint8 and buf.view(np.int16).tolist() == [1, 1, 1, -1, -1]
    out = np.zeros(5, dtype=np.float32)
    assert p.decompress(buf, out) == 0 and np.array_equal(out, f)
    for dtype, shape, eps in ((np.float32, (70_001,), 1e-3), (np.float64, (3, 1, 4_099), 0.5),
                              (np.float64, (1, 65_536), 1e-7), (np.float32, (257, 9), 1e-4)):
        p.set_options({"frsz:epsilon": eps})
        x = workloads.normal_np(int(np.prod(shape)), dtype, seed=11).reshape(shape) * dtype(10.0)
        n = legacy.legacy_length(shape)
        want = oracle.frsz1_compress(np.ascontiguousarray(x).reshape(-1)[:n], eps)
        yw = oracle.frsz1_decompress(want, dtype, eps)
        uint = np.uint64 if dtype == np.float64 else np.uint32
        rc, hbuf = p.compress(x)
        assert rc == 0 and np.array_equal(hbuf.view(np.int16), want), (dtype, shape)
        rc, dbuf = p.compress(torch.from_numpy(x).cuda())
        assert rc == 0 and dbuf.dtype == torch.uint8 and np.array_equal(dbuf.cpu().numpy(), hbuf)
        host_out = np.full(shape, -1.0, dtype=dtype)
        assert p.decompress(hbuf, host_out) == 0
        assert np.array_equal(host_out.reshape(-1)[:n].view(uint), yw.view(uint))
        assert np.all(host_out.reshape(-1)[n:] == -1.0)
        dev_out = torch.full(shape, -1.0, dtype=torch.from_numpy(x).dtype, device="cuda")
        assert p.decompress(dbuf, dev_out) == 0
        assert np.array_equal(dev_out.cpu().numpy().reshape(-1).view(uint), host_out.reshape(-1).view(uint))
    p.set_options({"frsz:epsilon": 0.0})
    assert p.compress(f)[0] == 2 and p.error_code == 2


@pytest.mark.gpu
def test_gpu_rounding_ties_and_edges(cuda):
    """Ties of the quantizer's round-half-away, magnitudes past 2^52 (already
    integers), signed zeros, subnormals and differences at the int16 limits,
    in both float types: bit for bit against the oracle (C round)."""
    rng = np.random.default_rng(17)
    for dtype in (np.float32, np.float64):
        k = rng.integers(-40_000, 40_000, 3000).astype(np.float64)
        parts = [k + 0.5, k - 0.5, -(k + 0.5), k,                  # ties at epsilon 0.5 (step 1)
                 np.array([0.5, -0.5, 1.5, -1.5, 2.5, -2.5, 0.49999997, -0.49999997, 0.0, -0.0]),
                 np.array([2.0 ** 52, -(2.0 ** 52) - 2, 2.0 ** 53 + 2, 1e20, -1e20, 3e38, -3e38]),
                 np.array([1e-40, -1e-45, 5e-324 if dtype == np.float64 else 1e-45]),
                 np.array([32767.5, -32768.5, 32766.5, -32767.5, 65535.0, -65536.0])]
        x = np.concatenate(parts).astype(dtype)
        x = np.concatenate([x, np.cumsum(rng.choice([-32768.0, 32767.0, 32767.5, -32768.5], 600)).astype(dtype)])
        t = torch.from_numpy(x).cuda()
        for eps in (0.5, 0.25, 1e-3):
            with np.errstate(over="ignore", invalid="ignore"):
                want = oracle.frsz1_compress(x, eps)
            got = legacy.compress(t, eps).cpu().numpy()
            assert np.array_equal(got, want), (dtype, eps, np.nonzero(got != want)[0][:5])
