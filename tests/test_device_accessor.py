"""The device accessor frsz::frsz2_compressor::decompress_gpu_element
(include/frsz2_b200_device.cuh), called from the test's own kernels: on CPU
the header compiles with nvcc for sm_100a; on a GPU every value it reads,
for every instance in tests/cuda/frsz2_accessor_test.cu, equals the oracle's
decoded value bit for bit (special values included) and the library's
frsz2_decompress_elements."""
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
SRC = os.path.join(ROOT, "tests", "cuda", "frsz2_accessor_test.cu")
LIBDIR = os.path.join(ROOT, "frsz_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_accessor_lib(out_dir: str) -> str:
    so = os.path.join(out_dir, "libfrsz2_accessor_test.so")
    subprocess.run([os.path.join(CUDA, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                    "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"), SRC,
                    "-o", so, "-L", LIBDIR, "-lfrsz2_b200", f"-Xlinker=-rpath,{LIBDIR}"], check=True)
    return so


@pytest.fixture(scope="module")
def accessor_lib(tmp_path_factory):
    frsz_b200.lib()  # the library the test links against is built
    lib = ctypes.CDLL(build_accessor_lib(str(tmp_path_factory.mktemp("accessor"))))
    lib.frsz2_accessor_test_decode.restype = ctypes.c_int
    lib.frsz2_accessor_test_decode.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                               ctypes.c_void_p]
    return lib


def cases(lib):
    cap = 64
    a, b, c = (ctypes.c_int * cap)(), (ctypes.c_int * cap)(), (ctypes.c_int * cap)()
    k = lib.frsz2_accessor_test_cases(a, b, c, cap)
    return [(bool(a[i]), b[i], c[i]) for i in range(k)]


def test_accessor_header_compiles(accessor_lib):
    assert len(cases(accessor_lib)) == 21


def values_with_specials(dtype, n, bits, seed):
    rng = np.random.default_rng(seed)
    lo, hi = (-30, 30) if dtype == np.float64 and bits <= 8 else (-20, 20)
    x = workloads.loguniform_np(n, dtype, seed=seed, lo=lo, hi=hi)
    fi = np.finfo(dtype)
    pick = rng.choice(n, n // 10, replace=False)
    kinds = rng.integers(0, 6, pick.size)
    x[pick[kinds == 0]] = 0.0
    x[pick[kinds == 1]] = -0.0
    x[pick[kinds == 2]] = (rng.random((kinds == 2).sum()) * float(fi.tiny)).astype(dtype)  # subnormal
    x[pick[kinds == 3]] = np.inf
    x[pick[kinds == 4]] = np.nan
    x[pick[kinds == 5]] = -np.inf
    # one whole block of tiny values (exponent far below the normal range of
    # the decoded fixed point)
    x[:64] = (rng.standard_normal(64) * float(fi.tiny) * 8).astype(dtype)
    return x


@pytest.mark.gpu
def test_accessor_matches_oracle(cuda, accessor_lib):
    for is64, bits, E in cases(accessor_lib):
        dtype = np.float64 if is64 else np.float32
        n = 3 * E + 1000 + 7
        x = values_with_specials(dtype, n, bits, seed=bits * 131 + E)
        ref = oracle.compress(x, bits, E)
        want = oracle.decompress(ref, n, dtype, bits, E)
        buf = torch.from_numpy(ref).cuda()
        idx = torch.cat([torch.arange(n, dtype=torch.int64),
                         torch.from_numpy(np.random.default_rng(bits).permutation(n))]).cuda()
        tdt = torch.float64 if is64 else torch.float32
        out = torch.full((idx.numel(),), float("nan"), dtype=tdt, device="cuda")
        rc = accessor_lib.frsz2_accessor_test_decode(int(is64), bits, E, buf.data_ptr(), n, idx.data_ptr(),
                                                     idx.numel(), out.data_ptr(),
                                                     torch.cuda.current_stream().cuda_stream)
        assert rc == 0, (is64, bits, E, rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        uint = np.uint64 if is64 else np.uint32
        exp = want[idx.cpu().numpy()]
        bad = np.nonzero(got.view(uint) != exp.view(uint))[0]
        assert bad.size == 0, f"{dtype.__name__} bits={bits} E={E}: {bad.size} values differ, first at {bad[:4]}"
        lib_out = frsz_b200.decompress_elements(buf, n, tdt, bits, E, idx)
        assert np.array_equal(lib_out.cpu().numpy().view(uint), got.view(uint)), (is64, bits, E)
