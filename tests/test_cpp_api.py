"""The C++ drop-in headers: they compile against the C ABI here (CPU), and
on a GPU the test program's compress_cpu_impl bytes equal the reference's
own bytes for the reference test's end-to-end cases."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "frsz2_api_test.cpp")
LIBDIR = os.path.join(ROOT, "frsz_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_test_program(out_dir: str) -> str:
    exe = os.path.join(out_dir, "frsz2_api_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(CUDA, "include"), SRC, "-o", exe, "-L", LIBDIR, "-lfrsz2_b200",
                    "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{LIBDIR}",
                    f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"], check=True)
    return exe


def test_headers_compile_and_link(tmp_path):
    import frsz_b200

    frsz_b200.lib()
    assert os.path.exists(build_test_program(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_api_on_gpu(tmp_path, cuda):
    exe = build_test_program(str(tmp_path))
    out = tmp_path / "e2e.bin"
    r = subprocess.run([exe, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    golden = np.load(os.path.join(ROOT, "tests", "golden", "e2e_reference_test.npz"))
    data = out.read_bytes()
    pos = 0
    seen = 0
    while pos < len(data):
        es, bits, E, size = np.frombuffer(data[pos:pos + 16], dtype=np.uint32)
        pos += 16
        buf = np.frombuffer(data[pos:pos + size], dtype=np.uint8)
        pos += int(size)
        key = f"{'float64' if es == 8 else 'float32'}_b{bits}_e{E}"
        assert np.array_equal(buf, golden[key]), key
        seen += 1
    assert seen == 11
