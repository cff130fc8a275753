"""CPU checkers for the FRSZ2 codec -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg /
``--impl reference`` arm of ``bench.py`` may import this package.  The product
(``frsz_b200``) never imports it and has no CPU fallback.

Two libraries, both built by ``oracle/Makefile``:

* ``libfrsz2_oracle.so`` -- ``frsz2_oracle.c``, a plain-C restatement of the
  reference codec (robertu94/frsz ``include/frsz2.hpp``) with bits / block size /
  float type as runtime arguments.
* ``_ref/libfrsz2_ref.so`` -- the reference's own ``frsz2.hpp`` compiled
  unmodified behind ``ref_shim.cpp``.  Present where it was built (it travels
  with the repository snapshot as a git-ignored binary).
* ``_ref/libfrsz2_ref_gpu.so`` -- the reference's own GPU kernels
  (``compress_gpu`` / ``decompress_gpu``) behind ``ref_gpu_shim.cu``, a speed bar
  for the GPU tests (not a checker: their zero-code decode differs from the
  reference CPU codec).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libfrsz2_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfrsz2_ref.so")

_c_size = ctypes.c_size_t
_vp = ctypes.c_void_p


def reference_dir() -> str:
    """The reference checkout: $FRSZ_REF_DIR, else a `reference` directory
    beside the repository (the Makefile's rule)."""
    return os.environ.get("FRSZ_REF_DIR") or os.path.abspath(os.path.join(HERE, os.pardir, os.pardir, "reference"))


def build(with_reference: bool = True) -> None:
    """Compile the restatement (and, where the reference sources exist, the
    reference shim).  Uses the committed Makefile."""
    target = "all" if with_reference else os.path.join(HERE, "libfrsz2_oracle.so")
    subprocess.run(["make", "-s", "-C", HERE, f"REF_DIR={reference_dir()}", target], check=True)


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


class _Lib:
    def __init__(self, path: str, prefix: str):
        self.path = path
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(with_reference=False)
        lib = ctypes.CDLL(ORACLE_SO)
        lib.frsz2o_word_bits.argtypes = [ctypes.c_int]
        lib.frsz2o_block_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.frsz2o_block_bytes.restype = _c_size
        lib.frsz2o_exponent_bytes.argtypes = [ctypes.c_int, ctypes.c_int, _c_size]
        lib.frsz2o_exponent_bytes.restype = _c_size
        lib.frsz2o_compressed_bytes.argtypes = [ctypes.c_int, ctypes.c_int, _c_size]
        lib.frsz2o_compressed_bytes.restype = _c_size
        for t, ft, ut in (("f32", ctypes.c_float, ctypes.c_uint32), ("f64", ctypes.c_double, ctypes.c_uint64)):
            getattr(lib, f"frsz2o_exponent_{t}").argtypes = [ft]
            getattr(lib, f"frsz2o_significand_{t}").argtypes = [ft]
            getattr(lib, f"frsz2o_significand_{t}").restype = ut
            getattr(lib, f"frsz2o_sign_{t}").argtypes = [ft]
            getattr(lib, f"frsz2o_floating_to_fixed_{t}").argtypes = [ft, ctypes.c_int16]
            getattr(lib, f"frsz2o_floating_to_fixed_{t}").restype = ut
            getattr(lib, f"frsz2o_fixed_to_floating_{t}").argtypes = [ut, ctypes.c_int64]
            getattr(lib, f"frsz2o_fixed_to_floating_{t}").restype = ft
            getattr(lib, f"frsz2o_compress_{t}").argtypes = [_vp, _c_size, ctypes.c_int, ctypes.c_int, _vp]
            getattr(lib, f"frsz2o_decompress_{t}").argtypes = [_vp, _c_size, ctypes.c_int, ctypes.c_int, _vp]
            getattr(lib, f"frsz2o_decompress_element_{t}").argtypes = [_vp, _c_size, ctypes.c_int, ctypes.c_int, _c_size]
            getattr(lib, f"frsz2o_decompress_element_{t}").restype = ft
        lib.frsz2o_compress_mt.argtypes = [ctypes.c_int, _vp, _c_size, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int]
        lib.frsz2o_decompress_mt.argtypes = [ctypes.c_int, _vp, _c_size, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int]
        for t in ("f32", "f64"):
            getattr(lib, f"frsz1o_compress_{t}").argtypes = [_vp, _c_size, ctypes.c_double, _vp]
            getattr(lib, f"frsz1o_compress_{t}").restype = None
            getattr(lib, f"frsz1o_decompress_{t}").argtypes = [_vp, _c_size, ctypes.c_double, ctypes.c_int, _vp]
            getattr(lib, f"frsz1o_decompress_{t}").restype = None
        _oracle = lib
    return _oracle


REF_GPU_SO = os.path.join(HERE, "_ref", "libfrsz2_ref_gpu.so")
_ref_gpu = None


def ref_gpu_lib():
    """The reference's own GPU kernels (compress_gpu / decompress_gpu) for the
    benchmark configurations; speed bar only, not the oracle."""
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(REF_GPU_SO):
            raise FileNotFoundError(f"{REF_GPU_SO} not built (needs the reference sources; see oracle/Makefile)")
        lib = ctypes.CDLL(REF_GPU_SO)
        lib.frsz2ref_gpu.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _c_size, _vp, _vp]
        _ref_gpu = lib
    return _ref_gpu


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources; see oracle/Makefile)")
        lib = ctypes.CDLL(REF_SO)
        lib.frsz2ref_compress.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _c_size, _vp, ctypes.c_int]
        lib.frsz2ref_decompress.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _c_size, _vp, ctypes.c_int]
        lib.frsz2ref_decompress_element_f64.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _c_size, _c_size]
        lib.frsz2ref_decompress_element_f64.restype = ctypes.c_double
        lib.frsz2ref_decompress_element_f32.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _c_size, _c_size]
        lib.frsz2ref_decompress_element_f32.restype = ctypes.c_float
        lib.frsz2ref_sizes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_size,
                                       ctypes.POINTER(_c_size), ctypes.POINTER(_c_size)]
        for t, ft, ut in (("f32", ctypes.c_float, ctypes.c_uint32), ("f64", ctypes.c_double, ctypes.c_uint64)):
            getattr(lib, f"frsz2ref_exponent_{t}").argtypes = [ft]
            getattr(lib, f"frsz2ref_significand_{t}").argtypes = [ft]
            getattr(lib, f"frsz2ref_significand_{t}").restype = ut
            getattr(lib, f"frsz2ref_sign_{t}").argtypes = [ft]
            getattr(lib, f"frsz2ref_floating_to_fixed_{t}").argtypes = [ft, ctypes.c_int16]
            getattr(lib, f"frsz2ref_floating_to_fixed_{t}").restype = ut
            getattr(lib, f"frsz2ref_fixed_to_floating_{t}").argtypes = [ut, ctypes.c_int16]
            getattr(lib, f"frsz2ref_fixed_to_floating_{t}").restype = ft
        _ref = lib
    return _ref


# ----------------------------------------------------------------- size algebra

def word_bits(bits: int) -> int:
    return 8 if bits <= 8 else 16 if bits <= 16 else 32 if bits <= 32 else 64


def compressed_bytes(bits: int, block_size: int, n: int) -> int:
    return int(oracle_lib().frsz2o_compressed_bytes(bits, block_size, n))


def exponent_bytes(bits: int, block_size: int, n: int) -> int:
    return int(oracle_lib().frsz2o_exponent_bytes(bits, block_size, n))


def block_bytes(bits: int, block_size: int) -> int:
    return int(oracle_lib().frsz2o_block_bytes(bits, block_size))


# ----------------------------------------------------------------- codecs

def _tag(a_dtype) -> str:
    d = np.dtype(a_dtype)
    if d == np.float32:
        return "f32"
    if d == np.float64:
        return "f64"
    raise TypeError(f"unsupported dtype {d}")


def compress(x: np.ndarray, bits: int, block_size: int, canary: int = 0xFF, threads: int = 1) -> np.ndarray:
    """Oracle compress into a canary-prefilled buffer of exactly
    compute_compressed_memory_size_byte(n) bytes."""
    x = np.ascontiguousarray(x)
    n = x.size
    out = np.full(compressed_bytes(bits, block_size, n), canary, dtype=np.uint8)
    lib = oracle_lib()
    if threads > 1:
        rc = lib.frsz2o_compress_mt(int(x.dtype == np.float64), _np_ptr(x), n, bits, block_size, _np_ptr(out), threads)
    else:
        rc = getattr(lib, f"frsz2o_compress_{_tag(x.dtype)}")(_np_ptr(x), n, bits, block_size, _np_ptr(out))
    if rc != 0:
        raise RuntimeError(f"oracle compress failed ({rc})")
    return out


def decompress(buf: np.ndarray, n: int, dtype, bits: int, block_size: int, threads: int = 1) -> np.ndarray:
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    out = np.empty(n, dtype=dtype)
    lib = oracle_lib()
    if threads > 1:
        rc = lib.frsz2o_decompress_mt(int(np.dtype(dtype) == np.float64), _np_ptr(buf), n, bits, block_size,
                                      _np_ptr(out), threads)
    else:
        rc = getattr(lib, f"frsz2o_decompress_{_tag(dtype)}")(_np_ptr(buf), n, bits, block_size, _np_ptr(out))
    if rc != 0:
        raise RuntimeError(f"oracle decompress failed ({rc})")
    return out


def decompress_element(buf: np.ndarray, n: int, dtype, bits: int, block_size: int, idx: int) -> float:
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    return getattr(oracle_lib(), f"frsz2o_decompress_element_{_tag(dtype)}")(_np_ptr(buf), n, bits, block_size, idx)


def ref_compress(x: np.ndarray, bits: int, block_size: int, canary: int = 0xFF, threads: int = 1) -> np.ndarray:
    """The reference's own compress_cpu_impl (threads == 1) or its
    compress_cpu_block over thread-split block ranges."""
    x = np.ascontiguousarray(x)
    n = x.size
    out = np.full(compressed_bytes(bits, block_size, n), canary, dtype=np.uint8)
    rc = ref_lib().frsz2ref_compress(int(x.dtype == np.float64), bits, block_size, _np_ptr(x), n, _np_ptr(out), threads)
    if rc != 0:
        raise RuntimeError(f"reference has no instance for bits={bits} E={block_size}")
    return out


def ref_decompress(buf: np.ndarray, n: int, dtype, bits: int, block_size: int, threads: int = 1) -> np.ndarray:
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    out = np.empty(n, dtype=dtype)
    rc = ref_lib().frsz2ref_decompress(int(np.dtype(dtype) == np.float64), bits, block_size, _np_ptr(buf), n,
                                       _np_ptr(out), threads)
    if rc != 0:
        raise RuntimeError(f"reference has no instance for bits={bits} E={block_size}")
    return out


def ref_compress_into(x: np.ndarray, out: np.ndarray, bits: int, block_size: int, threads: int = 1) -> None:
    rc = ref_lib().frsz2ref_compress(int(x.dtype == np.float64), bits, block_size, _np_ptr(x), x.size, _np_ptr(out),
                                     threads)
    if rc != 0:
        raise RuntimeError("reference compress failed")


def ref_decompress_into(buf: np.ndarray, out: np.ndarray, bits: int, block_size: int, threads: int = 1) -> None:
    rc = ref_lib().frsz2ref_decompress(int(out.dtype == np.float64), bits, block_size, _np_ptr(buf), out.size,
                                       _np_ptr(out), threads)
    if rc != 0:
        raise RuntimeError("reference decompress failed")


def error_bound(block_exponents: np.ndarray, bits: int) -> np.ndarray:
    """Per-block absolute error bound |x - x_hat| < 2^(e_b - bits + 2), widened
    by the zero rule 2^(e_b - 31) (truncation in floating_to_fixed,
    frsz2.hpp:361-370, and uint_fp_to_compressed, frsz2.hpp:555-558)."""
    e = block_exponents.astype(np.float64)
    return np.maximum(np.exp2(e - bits + 2), np.exp2(e - 31))


# ---------------------------------------------------------------- legacy "frsz"

def frsz1_compress(x: np.ndarray, epsilon: float) -> np.ndarray:
    """The legacy codec's int16 stream of x (src/frsz.cc:103-130)."""
    x = np.ascontiguousarray(x)
    out = np.empty(x.size, dtype=np.int16)
    t = "f64" if x.dtype == np.float64 else "f32"
    getattr(oracle_lib(), f"frsz1o_compress_{t}")(_np_ptr(x), x.size, float(epsilon), _np_ptr(out))
    return out


def frsz1_decompress(q: np.ndarray, dtype, epsilon: float, own_deltas: bool = False) -> np.ndarray:
    """The legacy codec's values from its int16 stream (src/frsz.cc:132-150);
    own_deltas=False reproduces the reference's use of block 0's deltas."""
    q = np.ascontiguousarray(q, dtype=np.int16)
    out = np.empty(q.size, dtype=dtype)
    t = "f64" if np.dtype(dtype) == np.float64 else "f32"
    getattr(oracle_lib(), f"frsz1o_decompress_{t}")(_np_ptr(q), q.size, float(epsilon), int(own_deltas),
                                                   _np_ptr(out))
    return out
