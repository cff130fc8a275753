"""ctypes binding of libfrsz2_b200.so (the C ABI declared in include/frsz2_b200.h).

There is no fallback: if the library is missing or fails to load, every call
raises.  Build it with ``python -m frsz_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfrsz2_b200.so")

FRSZ2_OK = 0
FRSZ2_EDTYPE = 1
FRSZ2_EFAIL = 2
FRSZ2_FLOAT = 0
FRSZ2_DOUBLE = 1

_u64 = ctypes.c_uint64
_vp = ctypes.c_void_p
_int = ctypes.c_int

class BatchItemC(ctypes.Structure):
    """frsz2_batch_item (include/frsz2_b200.h)."""
    _fields_ = [("dtype", ctypes.c_int), ("bits", ctypes.c_int), ("block_size", ctypes.c_int),
                ("n", ctypes.c_uint64), ("values", ctypes.c_void_p), ("decompressed", ctypes.c_void_p),
                ("compressed", ctypes.c_void_p)]


class BatchStatsC(ctypes.Structure):
    """frsz2_batch_stats (include/frsz2_b200.h)."""
    _fields_ = [("arrays", ctypes.c_uint64), ("persistent_arrays", ctypes.c_uint64),
                ("separate_launches", ctypes.c_uint64), ("classes", ctypes.c_uint64),
                ("tiles", ctypes.c_uint64 * 2), ("threads_per_cta", ctypes.c_int * 2),
                ("rows_per_warp", ctypes.c_int * 2), ("ctas_per_sm", ctypes.c_int * 2),
                ("side_by_side", ctypes.c_int * 2), ("tuned", ctypes.c_int * 2),
                ("one_cta_per_tile", ctypes.c_int * 2)]


class RequestC(ctypes.Structure):
    """frsz2_request (include/frsz2_b200.h)."""
    _fields_ = [("op", ctypes.c_int), ("dtype", ctypes.c_int), ("bits", ctypes.c_int), ("block_size", ctypes.c_int),
                ("n", ctypes.c_uint64), ("input", ctypes.c_void_p), ("output", ctypes.c_void_p),
                ("arrival_ns", ctypes.c_uint64), ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class CompletionC(ctypes.Structure):
    """frsz2_completion (include/frsz2_b200.h)."""
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int), ("op", ctypes.c_int), ("output", ctypes.c_void_p),
                ("output_bytes", ctypes.c_uint64), ("bytes", ctypes.c_uint64), ("arrival_ns", ctypes.c_uint64),
                ("admit_ns", ctypes.c_uint64), ("done_ns", ctypes.c_uint64)]


class CountersC(ctypes.Structure):
    """frsz2_server_counters (include/frsz2_b200.h)."""
    _fields_ = [(k, ctypes.c_uint64) for k in ("completed", "failed", "batches", "bytes", "pending", "budget_bytes",
                                               "arena_used_bytes", "arena_peak_bytes", "max_batch",
                                               "max_inflight_output_bytes")]


# name -> (restype, argtypes); kept in step with include/frsz2_b200.h
SIGNATURES = {
    "register_frsz": (None, []),
    "frsz2_version": (ctypes.c_char_p, []),
    "frsz2_last_error": (ctypes.c_char_p, []),
    "frsz2_compressed_size": (_int, [_int, _int, _int, _u64, ctypes.POINTER(_u64)]),
    "frsz2_exponent_size": (_int, [_int, _int, _int, _u64, ctypes.POINTER(_u64)]),
    "frsz2_compress": (_int, [_int, _int, _int, _vp, _u64, _vp, _vp]),
    "frsz2_decompress": (_int, [_int, _int, _int, _vp, _u64, _vp, _vp]),
    "frsz2_compress_host": (_int, [_int, _int, _int, _vp, _u64, _vp, _vp]),
    "frsz2_decompress_host": (_int, [_int, _int, _int, _vp, _u64, _vp, _vp]),
    "frsz2_decompress_elements": (_int, [_int, _int, _int, _vp, _u64, _vp, _u64, _vp, _vp]),
    "frsz2_decompress_elements_host": (_int, [_int, _int, _int, _vp, _u64, _vp, _u64, _vp]),
    "frsz1_compressed_size": (_u64, [_u64]),
    "frsz1_compress": (_int, [_int, ctypes.c_double, _vp, _u64, _vp, _vp]),
    "frsz1_decompress": (_int, [_int, ctypes.c_double, _vp, _u64, _vp, _int, _vp]),
    "frsz2_compress_blocks": (_int, [_int, _int, _int, _vp, _u64, _u64, _u64, _vp, _vp]),
    "frsz2_decompress_blocks": (_int, [_int, _int, _int, _vp, _u64, _u64, _u64, _vp, _vp]),
    "frsz2_batch_create": (_int, [ctypes.POINTER(BatchItemC), _u64, ctypes.POINTER(_vp)]),
    "frsz2_batch_compress": (_int, [_vp, _vp]),
    "frsz2_batch_decompress": (_int, [_vp, _vp]),
    "frsz2_batch_autotune": (_int, [_vp, _int, _vp, ctypes.POINTER(ctypes.c_float)]),
    "frsz2_batch_configure": (_int, [_vp, _int, _int, _int, _int, _int]),
    "frsz2_batch_info": (_int, [_vp, ctypes.POINTER(BatchStatsC)]),
    "frsz2_batch_destroy": (None, [_vp]),
    "frsz2_batch_compress_static": (_int, [ctypes.POINTER(BatchItemC), _u64, _vp]),
    "frsz2_basis_workspace_size": (_u64, [_int, _u64]),
    "frsz2_basis_dot": (_int, [_int, _int, _int, ctypes.POINTER(_vp), _int, _u64, _vp, _vp, _vp, _u64, _vp]),
    "frsz2_basis_axpy": (_int, [_int, _int, _int, ctypes.POINTER(_vp), _int, _u64, _vp, _vp, _vp]),
    "frsz2_now_ns": (_u64, []),
    "frsz2_server_create": (_int, [_u64, _int, _int, ctypes.POINTER(_vp)]),
    "frsz2_server_submit": (_int, [_vp, ctypes.POINTER(RequestC), _u64, ctypes.POINTER(_u64)]),
    "frsz2_server_cancel": (_int, [_vp, _u64]),
    "frsz2_server_poll": (_int, [_vp, ctypes.POINTER(CompletionC), _u64, ctypes.POINTER(_u64), _int]),
    "frsz2_server_release": (_int, [_vp, _u64]),
    "frsz2_server_stats": (_int, [_vp, ctypes.POINTER(CountersC)]),
    "frsz2_server_destroy": (None, [_vp]),
}


class Frsz2Error(RuntimeError):
    """Non-zero status from the C ABI: 1 = unsupported dtype, 2 = unsupported
    bits / block size or runtime failure (src/frsz2.cc:164-168 semantics)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_lock = threading.Lock()
_handle = None


def lib() -> ctypes.CDLL:
    global _handle
    if _handle is None:
        with _lock:
            if _handle is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(f"{LIB_PATH} is not built; run `python -m frsz_b200.build` "
                                       "(the FRSZ2 codec has no CPU fallback)")
                h = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    fn = getattr(h, name)
                    fn.restype = res
                    fn.argtypes = args
                _handle = h
    return _handle


def check(rc: int) -> None:
    if rc != FRSZ2_OK:
        msg = lib().frsz2_last_error()
        raise Frsz2Error(rc, msg.decode() if msg else f"status {rc}")
