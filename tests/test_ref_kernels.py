"""The reference's launchable kernels frsz::compress_gpu / frsz::decompress_gpu
(include/frsz2.hpp:1258-1288) as the drop-in header provides them
(include/frsz2_b200.hpp), launched from an nvcc-built test library with the
reference test's own launch shapes.  On CPU the header compiles for sm_100a;
on a GPU the compressed buffers (0xFF canary, 128 bytes of slack) equal the
golden fixtures the reference produced for its end-to-end cases
(test/test_frsz_gpu.cu:382-410) byte for byte, the E = 1 lossless case round
trips, and the other instances equal the oracle, buffers and decoded
values."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cuda", "frsz2_ref_kernels_test.cu")
GOLDEN = os.path.join(ROOT, "tests", "golden")
LIBDIR = os.path.join(ROOT, "frsz_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SLACK = 128  # test/test_frsz_gpu.cu:333-335


@pytest.fixture(scope="module")
def refk_lib(tmp_path_factory):
    frsz_b200.lib()
    so = os.path.join(str(tmp_path_factory.mktemp("refk")), "libfrsz2_refk_test.so")
    subprocess.run([os.path.join(CUDA, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                    "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"), SRC,
                    "-o", so, "-L", LIBDIR, "-lfrsz2_b200", f"-Xlinker=-rpath,{LIBDIR}"], check=True)
    lib = ctypes.CDLL(so)
    lib.frsz2_refk_test_run.restype = ctypes.c_int
    lib.frsz2_refk_test_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return lib


def cases(lib):
    cap = 64
    a, b, c = (ctypes.c_int * cap)(), (ctypes.c_int * cap)(), (ctypes.c_int * cap)()
    k = lib.frsz2_refk_test_cases(a, b, c, cap)
    return [(bool(a[i]), b[i], c[i]) for i in range(k)]


def test_ref_kernels_header_compiles(refk_lib):
    assert len(cases(refk_lib)) == 18


def launch(lib, x: np.ndarray, bits: int, E: int):
    """Compressed buffer (+ slack) and decoded values from the two launches;
    the buffer starts as 0xFF and the output as +Inf, as in the reference's
    test (test/test_frsz_gpu.cu:332-335, 362)."""
    n = x.size
    size = frsz_b200.compressed_size(x.dtype, bits, E, n) + SLACK
    buf = torch.full((size,), 0xFF, dtype=torch.uint8, device="cuda")
    dx = torch.from_numpy(x).cuda()
    out = torch.full((n,), float("inf"), dtype=dx.dtype, device="cuda")
    rc = lib.frsz2_refk_test_run(int(x.dtype == np.float64), bits, E, dx.data_ptr(), n, buf.data_ptr(),
                                 out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, (x.dtype, bits, E, rc)
    torch.cuda.synchronize()
    return buf.cpu().numpy(), out.cpu().numpy()


@pytest.mark.gpu
def test_reference_end_to_end_cases_equal_golden(cuda, refk_lib):
    """The reference test's 11 end-to-end cases: n = 2049 (fp64) and 2160
    (fp32) values of its repeating pattern."""
    golden = np.load(os.path.join(GOLDEN, "e2e_reference_test.npz"))
    for key in golden.files:
        dt, b, e = key.split("_")
        dtype, bits, E = np.dtype(dt), int(b[1:]), int(e[1:])
        n = 2049 if dtype == np.float64 else 2160
        x = workloads.reference_pattern(n, dtype)
        got, y = launch(refk_lib, x, bits, E)
        assert np.array_equal(got, golden[key]), key
        want = oracle.decompress(golden[key][:-SLACK], n, dtype, bits, E)
        uint = np.uint64 if dtype == np.float64 else np.uint32
        assert np.array_equal(y.view(uint), want.view(uint)), key


@pytest.mark.gpu
def test_reference_lossless_case(cuda, refk_lib):
    """E = 1 at 32 bits round trips fp32 values exactly (test/test_frsz_gpu.cu:422-441)."""
    x = np.random.default_rng(4).uniform(-1e8, 1e8, 100_000).astype(np.float32)
    got, y = launch(refk_lib, x, 32, 1)
    assert np.array_equal(got[:-SLACK], oracle.compress(x, 32, 1)) and np.all(got[-SLACK:] == 0xFF)
    assert np.array_equal(y, x)


@pytest.mark.gpu
def test_other_instances_equal_oracle(cuda, refk_lib):
    for is64, bits, E in cases(refk_lib):
        dtype = np.float64 if is64 else np.float32
        for n in (1, E + 1, 4099):
            lo, hi = (-30, 30) if is64 and bits <= 8 else (-20, 20)
            x = workloads.loguniform_np(n, dtype, seed=bits * 7 + E + n, lo=lo, hi=hi)
            if n > 100:
                x[[3, 50, 77]] = [np.nan, np.inf, -0.0]
            got, y = launch(refk_lib, x, bits, E)
            ref = oracle.compress(x, bits, E, canary=0xFF)
            assert np.array_equal(got[:-SLACK], ref) and np.all(got[-SLACK:] == 0xFF), (dtype, bits, E, n)
            uint = np.uint64 if is64 else np.uint32
            want = oracle.decompress(ref, n, dtype, bits, E)
            assert np.array_equal(y.view(uint), want.view(uint)), (dtype, bits, E, n)
