"""Host-side mirror of the reference's FRSZ2 codec API over the C ABI.

``Frsz2Compressor`` mirrors ``frsz::frsz2_compressor<bits_per_value,
max_exp_block_size, FpType>`` (robertu94/frsz include/frsz2.hpp:504-1256): a
non-owning view of one compressed buffer with the same size functions and
accessors.  Its compress / decompress run the sm_100a kernels of
libfrsz2_b200.so; device buffers are torch CUDA tensors, host buffers are
numpy arrays (the ``*_host`` calls copy inside the C ABI).

``dispatch_frsz2_compression`` / ``dispatch_frsz2_decompression`` mirror the
runtime dispatch of include/frsz2.hpp:1292-1347: the caller names the
supported bit widths and block sizes and an unsupported value raises
``Frsz2Error`` with the reference's message.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Optional

import numpy as np
import torch

from ._lib import FRSZ2_DOUBLE, FRSZ2_EFAIL, FRSZ2_FLOAT, Frsz2Error, check, lib

_TORCH_DT = {torch.float32: FRSZ2_FLOAT, torch.float64: FRSZ2_DOUBLE}
_NP_DT = {np.dtype(np.float32): FRSZ2_FLOAT, np.dtype(np.float64): FRSZ2_DOUBLE}


def dtype_code(dtype) -> int:
    """FRSZ2_FLOAT / FRSZ2_DOUBLE for a torch or numpy dtype; raises
    Frsz2Error(1, "unsupported dtype") otherwise (src/frsz2.cc:164)."""
    if isinstance(dtype, torch.dtype):
        code = _TORCH_DT.get(dtype)
    else:
        try:
            code = _NP_DT.get(np.dtype(dtype))
        except TypeError:
            code = None
    if code is None:
        raise Frsz2Error(1, "unsupported dtype")
    return code


def word_bits(bits: int) -> int:
    """storage_t<bits> width (include/frsz2.hpp:258-262)."""
    return 8 if bits <= 8 else 16 if bits <= 16 else 32 if bits <= 32 else 64


def compressed_size(dtype, bits: int, block_size: int, n: int) -> int:
    """compute_compressed_memory_size_byte (include/frsz2.hpp:542-548)."""
    out = ctypes.c_uint64()
    check(lib().frsz2_compressed_size(dtype_code(dtype), bits, block_size, n, ctypes.byref(out)))
    return out.value


def exponent_size(dtype, bits: int, block_size: int, n: int) -> int:
    """compute_exponent_block_size_byte (include/frsz2.hpp:534-540)."""
    out = ctypes.c_uint64()
    check(lib().frsz2_exponent_size(dtype_code(dtype), bits, block_size, n, ctypes.byref(out)))
    return out.value


def _stream_ptr(stream: Optional[torch.cuda.Stream]) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _require_cuda(t: torch.Tensor, what: str) -> None:
    if not t.is_cuda:
        raise Frsz2Error(FRSZ2_EFAIL, f"{what} must be a CUDA tensor")
    if not t.is_contiguous():
        raise Frsz2Error(FRSZ2_EFAIL, f"{what} must be contiguous")


# ------------------------------------------------------------------ device API

def compress(values: torch.Tensor, bits: int, block_size: int, out: Optional[torch.Tensor] = None,
             stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """Compress a CUDA float32/float64 tensor (flattened) into a uint8 CUDA
    buffer of compressed_size() bytes.  A caller-supplied `out` keeps the bytes
    the format leaves unwritten (pad, unused tail words)."""
    _require_cuda(values, "values")
    code = dtype_code(values.dtype)
    n = values.numel()
    size = compressed_size(values.dtype, bits, block_size, n)
    if out is None:
        out = torch.empty(size, dtype=torch.uint8, device=values.device)
    else:
        _require_cuda(out, "out")
        if out.dtype != torch.uint8 or out.numel() < size:
            raise Frsz2Error(FRSZ2_EFAIL, f"out must be a uint8 tensor of at least {size} bytes")
    check(lib().frsz2_compress(code, bits, block_size, values.data_ptr(), n, out.data_ptr(), _stream_ptr(stream)))
    return out


def decompress(compressed: torch.Tensor, n: int, dtype, bits: int, block_size: int,
               out: Optional[torch.Tensor] = None, stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """Decompress `n` values of `dtype` from a uint8 CUDA buffer."""
    _require_cuda(compressed, "compressed")
    code = dtype_code(dtype)
    size = compressed_size(dtype, bits, block_size, n)
    if compressed.numel() < size:
        raise Frsz2Error(FRSZ2_EFAIL, f"compressed buffer holds {compressed.numel()} bytes, needs {size}")
    tdt = torch.float32 if code == FRSZ2_FLOAT else torch.float64
    if out is None:
        out = torch.empty(n, dtype=tdt, device=compressed.device)
    else:
        _require_cuda(out, "out")
        if out.dtype != tdt or out.numel() < n:
            raise Frsz2Error(FRSZ2_EFAIL, "out has the wrong dtype or size")
    check(lib().frsz2_decompress(code, bits, block_size, compressed.data_ptr(), n, out.data_ptr(),
                                 _stream_ptr(stream)))
    return out


def decompress_elements(compressed: torch.Tensor, n: int, dtype, bits: int, block_size: int,
                        indices: torch.Tensor, out: Optional[torch.Tensor] = None,
                        stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """Random-access decode of the values at `indices` (int64 CUDA tensor)."""
    _require_cuda(compressed, "compressed")
    _require_cuda(indices, "indices")
    code = dtype_code(dtype)
    tdt = torch.float32 if code == FRSZ2_FLOAT else torch.float64
    idx = indices.to(torch.int64).contiguous()
    if out is None:
        out = torch.empty(idx.numel(), dtype=tdt, device=compressed.device)
    check(lib().frsz2_decompress_elements(code, bits, block_size, compressed.data_ptr(), n, idx.data_ptr(),
                                          idx.numel(), out.data_ptr(), _stream_ptr(stream)))
    return out


# ------------------------------------------------------------------ host API

def compress_host(values: np.ndarray, bits: int, block_size: int, out: Optional[np.ndarray] = None,
                  stream: Optional[torch.cuda.Stream] = None) -> np.ndarray:
    """Host buffers in and out; copies and kernels run inside the call."""
    values = np.ascontiguousarray(values)
    code = dtype_code(values.dtype)
    size = compressed_size(values.dtype, bits, block_size, values.size)
    if out is None:
        out = np.zeros(size, dtype=np.uint8)
    check(lib().frsz2_compress_host(code, bits, block_size, values.ctypes.data, values.size, out.ctypes.data,
                                    _stream_ptr(stream)))
    return out


def decompress_host(compressed: np.ndarray, n: int, dtype, bits: int, block_size: int,
                    out: Optional[np.ndarray] = None, stream: Optional[torch.cuda.Stream] = None) -> np.ndarray:
    code = dtype_code(dtype)
    compressed = np.ascontiguousarray(compressed, dtype=np.uint8)
    if out is None:
        out = np.empty(n, dtype=np.float32 if code == FRSZ2_FLOAT else np.float64)
    check(lib().frsz2_decompress_host(code, bits, block_size, compressed.ctypes.data, n, out.ctypes.data,
                                      _stream_ptr(stream)))
    return out


def decompress_elements_host(compressed: np.ndarray, n: int, dtype, bits: int, block_size: int,
                             indices: np.ndarray, out: Optional[np.ndarray] = None) -> np.ndarray:
    """Random-access decode on host buffers (decompress_cpu_element,
    include/frsz2.hpp:1199-1214): the blocks holding the requested indices
    are decoded on the GPU.  Indices >= n leave their output untouched."""
    code = dtype_code(dtype)
    compressed = np.ascontiguousarray(compressed, dtype=np.uint8)
    idx = np.ascontiguousarray(indices, dtype=np.uint64)
    if out is None:
        out = np.zeros(idx.size, dtype=np.float32 if code == FRSZ2_FLOAT else np.float64)
    check(lib().frsz2_decompress_elements_host(code, bits, block_size, compressed.ctypes.data, n, idx.ctypes.data,
                                               idx.size, out.ctypes.data))
    return out


# ------------------------------------------------------------------ class view

class Frsz2Compressor:
    """View of one compressed buffer, mirroring
    frsz::frsz2_compressor<bits_per_value, max_exp_block_size, FpType>
    (include/frsz2.hpp:504-1256).  `buffer` is a uint8 CUDA tensor (device
    path) or numpy array (host path) of compute_compressed_memory_size_byte(n)
    bytes; the view never allocates it."""

    def __init__(self, bits_per_value: int, max_exp_block_size: int, fp_type, buffer, total_elements: int):
        self.bits_per_value = int(bits_per_value)
        self.max_exp_block_size = int(max_exp_block_size)
        self.fp_type = fp_type
        self._code = dtype_code(fp_type)
        if not 4 <= self.bits_per_value <= (32 if self._code == FRSZ2_FLOAT else 64):
            raise Frsz2Error(FRSZ2_EFAIL, f"Unsupported number of bits: {self.bits_per_value}")
        if self.max_exp_block_size <= 0:
            raise Frsz2Error(FRSZ2_EFAIL, f"Unsupported exponent block size: {self.max_exp_block_size}")
        self.buffer = buffer
        self.total_elements = int(total_elements)

    # static size algebra (include/frsz2.hpp:525-548)
    @property
    def uint_compressed_size_bit(self) -> int:
        return word_bits(self.bits_per_value)

    @property
    def compressed_block_size_element_count(self) -> int:
        w = self.uint_compressed_size_bit
        return -(-self.max_exp_block_size * self.bits_per_value // w)

    @property
    def compressed_block_size_byte(self) -> int:
        return self.compressed_block_size_element_count * self.uint_compressed_size_bit // 8

    def compute_exponent_block_size_byte(self, n: int) -> int:
        return exponent_size(self.fp_type, self.bits_per_value, self.max_exp_block_size, n)

    def compute_compressed_memory_size_byte(self, n: int) -> int:
        return compressed_size(self.fp_type, self.bits_per_value, self.max_exp_block_size, n)

    def get_total_elements(self) -> int:
        return self.total_elements

    def get_exponent_data(self):
        """exp_type[ceil(n/E)] view (include/frsz2.hpp:790-792)."""
        nb = -(-self.total_elements // self.max_exp_block_size)
        w = self.uint_compressed_size_bit // 8
        raw = self.buffer[: nb * w]
        if isinstance(raw, torch.Tensor):
            return raw.view({1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w])
        return raw.view({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[w])

    def get_compressed_data(self):
        """Word region (include/frsz2.hpp:786-788), as raw bytes."""
        return self.buffer[self.compute_exponent_block_size_byte(self.total_elements):]

    def compress_gpu_impl(self, values: torch.Tensor, stream=None) -> None:
        compress(values, self.bits_per_value, self.max_exp_block_size, out=self.buffer, stream=stream)

    def decompress_gpu_impl(self, out: torch.Tensor, stream=None) -> None:
        decompress(self.buffer, self.total_elements, self.fp_type, self.bits_per_value, self.max_exp_block_size,
                   out=out, stream=stream)

    def compress_host_impl(self, values: np.ndarray) -> None:
        """Host arrays, like the reference's compress_cpu_impl
        (include/frsz2.hpp:1181); the work runs on the GPU."""
        compress_host(values, self.bits_per_value, self.max_exp_block_size, out=self.buffer)

    def decompress_host_impl(self, out: np.ndarray) -> None:
        decompress_host(self.buffer, self.total_elements, self.fp_type, self.bits_per_value,
                        self.max_exp_block_size, out=out)

    def decompress_cpu_element(self, idx: int):
        """Value idx (include/frsz2.hpp:1199-1214); a host (numpy) buffer goes
        through the host-buffer call, a CUDA buffer through the device one."""
        if isinstance(self.buffer, torch.Tensor) and self.buffer.is_cuda:
            i = torch.tensor([idx], dtype=torch.int64, device=self.buffer.device)
            return self.decompress_gpu_elements(i).item()
        return decompress_elements_host(np.asarray(self.buffer), self.total_elements, self.fp_type,
                                        self.bits_per_value, self.max_exp_block_size,
                                        np.array([idx], dtype=np.uint64))[0]

    def decompress_gpu_elements(self, indices: torch.Tensor) -> torch.Tensor:
        """decompress_gpu_element (include/frsz2.hpp:1096-1104) for a batch
        of indices."""
        return decompress_elements(self.buffer, self.total_elements, self.fp_type, self.bits_per_value,
                                   self.max_exp_block_size, indices)


# ------------------------------------------------------------------ dispatch

def _dispatch(bit_list: Iterable[int], bits: int, exp_list: Iterable[int], block_size: int):
    if bits not in tuple(bit_list):
        raise Frsz2Error(FRSZ2_EFAIL, f"Unsupported number of bits: {bits}")
    if block_size not in tuple(exp_list):
        raise Frsz2Error(FRSZ2_EFAIL, f"Unsupported exponent block size: {block_size}")


def dispatch_frsz2_compression(fp_type, bit_list, bits: int, exp_list, block_size: int, data, total_elems: int,
                               comp_mem) -> None:
    """dispatch_frsz2_compression<FpType>(int_list_t<bits...>, bits,
    int_list_t<E...>, E, data, n, out) (include/frsz2.hpp:1346).  `data` and
    `comp_mem` are both CUDA tensors or both numpy arrays."""
    _dispatch(bit_list, bits, exp_list, block_size)
    c = Frsz2Compressor(bits, block_size, fp_type, comp_mem, total_elems)
    if isinstance(data, torch.Tensor):
        c.compress_gpu_impl(data[:total_elems])
    else:
        c.compress_host_impl(np.asarray(data)[:total_elems])


def dispatch_frsz2_decompression(fp_type, bit_list, bits: int, exp_list, block_size: int, data, total_elems: int,
                                 comp_mem) -> None:
    """dispatch_frsz2_decompression (include/frsz2.hpp:1347): fills `data`."""
    _dispatch(bit_list, bits, exp_list, block_size)
    c = Frsz2Compressor(bits, block_size, fp_type, comp_mem, total_elems)
    if isinstance(data, torch.Tensor):
        c.decompress_gpu_impl(data)
    else:
        c.decompress_host_impl(data)
