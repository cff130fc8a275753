"""Batched FRSZ2: many device arrays of mixed float types, widths, block sizes
and sizes per call, through the C ABI's frsz2_batch_* plan (one CUDA graph
launch of per-class persistent kernels, autotuned launch shape).  No
counterpart in the reference, which compresses one array per call."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import torch

from ._lib import BatchItemC, BatchStatsC, check, lib
from .codec import dtype_code


@dataclass
class BatchArray:
    """One array of a batch: `values` (compress input), `compressed` (uint8
    buffer of compressed_size() bytes) and `decompressed` (decompress output;
    defaults to `values`).  All CUDA tensors."""
    values: Optional[torch.Tensor]
    compressed: torch.Tensor
    bits: int
    block_size: int
    decompressed: Optional[torch.Tensor] = None
    n: Optional[int] = None


class BatchPlan:
    """Device-resident descriptors of a fixed set of arrays; compress() and
    decompress() each run as one graph launch.  The tensors must stay alive
    (and in place) as long as the plan."""

    def __init__(self, arrays: Sequence[BatchArray]):
        self.arrays: List[BatchArray] = list(arrays)
        items = (BatchItemC * max(1, len(self.arrays)))()
        for i, a in enumerate(self.arrays):
            ref = a.values if a.values is not None else a.decompressed
            out = a.decompressed if a.decompressed is not None else a.values
            n = a.n if a.n is not None else ref.numel()
            items[i].dtype = dtype_code(ref.dtype)
            items[i].bits = a.bits
            items[i].block_size = a.block_size
            items[i].n = n
            items[i].values = a.values.data_ptr() if a.values is not None else None
            items[i].decompressed = out.data_ptr() if out is not None else None
            items[i].compressed = a.compressed.data_ptr()
        self._items = items
        h = ctypes.c_void_p()
        check(lib().frsz2_batch_create(items, len(self.arrays), ctypes.byref(h)))
        self._h = h

    def _stream(self, stream):
        return (stream or torch.cuda.current_stream()).cuda_stream

    def compress(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        check(lib().frsz2_batch_compress(self._h, self._stream(stream)))

    def decompress(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        check(lib().frsz2_batch_decompress(self._h, self._stream(stream)))

    def autotune(self, compress: bool = True, stream: Optional[torch.cuda.Stream] = None) -> float:
        """Pick the fastest launch shape for one direction; returns its time (ms)."""
        ms = ctypes.c_float()
        check(lib().frsz2_batch_autotune(self._h, int(compress), self._stream(stream), ctypes.byref(ms)))
        return ms.value

    def configure(self, compress: bool, shape: int = 0, ctas_per_sm: int = 4, side_by_side: bool = False,
                  one_cta_per_tile: bool = False) -> None:
        """Set one direction's launch configuration by hand
        (frsz2_batch_configure)."""
        check(lib().frsz2_batch_configure(self._h, int(compress), shape, ctas_per_sm, int(side_by_side),
                                          int(one_cta_per_tile)))

    def info(self) -> dict:
        st = BatchStatsC()
        check(lib().frsz2_batch_info(self._h, ctypes.byref(st)))
        out = {k: getattr(st, k) for k in ("arrays", "persistent_arrays", "separate_launches", "classes")}
        for k in ("tiles", "threads_per_cta", "rows_per_warp", "ctas_per_sm", "side_by_side", "tuned",
                  "one_cta_per_tile"):
            v = getattr(st, k)
            out[k] = {"decompress": v[0], "compress": v[1]}
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().frsz2_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
