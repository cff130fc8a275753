"""A compressed fp64 vector basis (Krylov-style) with decompression fused
into its consumers: h = V^T w and y += V c read the FRSZ2 buffers directly
(frsz2_basis_dot / frsz2_basis_axpy), never materialising the vectors."""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from ._lib import FRSZ2_DOUBLE, check, lib
from . import codec


class CompressedBasis:
    def __init__(self, capacity: int, n: int, bits: int = 32, block_size: int = 32, device="cuda"):
        self.capacity, self.n, self.bits, self.block_size = capacity, n, bits, block_size
        size = codec.compressed_size(torch.float64, bits, block_size, n)
        self.buffers = [torch.zeros(size, dtype=torch.uint8, device=device) for _ in range(capacity)]
        self._ptrs = (ctypes.c_void_p * max(1, capacity))(*[b.data_ptr() for b in self.buffers])
        ws = lib().frsz2_basis_workspace_size(capacity, n)
        self.workspace = torch.zeros(ws, dtype=torch.uint8, device=device)
        self.size = 0

    def _stream(self, stream):
        return (stream or torch.cuda.current_stream()).cuda_stream

    def set(self, j: int, v: torch.Tensor, stream=None) -> None:
        codec.compress(v.to(torch.float64).contiguous(), self.bits, self.block_size, out=self.buffers[j],
                       stream=stream)
        self.size = max(self.size, j + 1)

    def append(self, v: torch.Tensor, stream=None) -> int:
        j = self.size
        self.set(j, v, stream)
        return j

    def get(self, j: int, stream=None) -> torch.Tensor:
        return codec.decompress(self.buffers[j], self.n, torch.float64, self.bits, self.block_size, stream=stream)

    def dot(self, w: torch.Tensor, m: Optional[int] = None, out: Optional[torch.Tensor] = None,
            stream=None) -> torch.Tensor:
        """h[j] = <V_j, w> for j < m."""
        m = self.size if m is None else m
        h = out if out is not None else torch.empty(m, dtype=torch.float64, device=w.device)
        check(lib().frsz2_basis_dot(FRSZ2_DOUBLE, self.bits, self.block_size, self._ptrs, m, self.n,
                                    w.data_ptr(), h.data_ptr(), self.workspace.data_ptr(), self.workspace.numel(),
                                    self._stream(stream)))
        return h

    def axpy(self, c: torch.Tensor, y: torch.Tensor, m: Optional[int] = None, stream=None) -> torch.Tensor:
        """y += sum_{j<m} c[j] V_j, in place."""
        m = self.size if m is None else m
        check(lib().frsz2_basis_axpy(FRSZ2_DOUBLE, self.bits, self.block_size, self._ptrs, m, self.n,
                                     c.data_ptr(), y.data_ptr(), self._stream(stream)))
        return y
