"""The reference's legacy "frsz" codec (the LibPressio plugin "frsz",
src/frsz.cc:15-165) on the GPU: epsilon quantization, int16 differences
within blocks of 256 values.  Device tensors in and out; the work runs in the
library's CUDA kernels (frsz_b200/csrc/frsz1_legacy.cu)."""
from __future__ import annotations

from typing import Optional

import torch

from ._lib import FRSZ2_EFAIL, FRSZ2_FLOAT, Frsz2Error, check, lib
from .codec import _require_cuda, _stream_ptr, dtype_code

FRSZ1_OWN_DELTAS = 1
DEFAULT_EPSILON = 1e-4  # "frsz:epsilon" (src/frsz.cc:152)


def compress(values: torch.Tensor, epsilon: float = DEFAULT_EPSILON, out: Optional[torch.Tensor] = None,
             stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """int16 stream of a CUDA float32 / float64 tensor (compress_1d,
    src/frsz.cc:103-130)."""
    _require_cuda(values, "values")
    n = values.numel()
    if out is None:
        out = torch.empty(n, dtype=torch.int16, device=values.device)
    elif out.dtype != torch.int16 or out.numel() < n:
        raise Frsz2Error(FRSZ2_EFAIL, "out must be an int16 tensor of at least n elements")
    check(lib().frsz1_compress(dtype_code(values.dtype), float(epsilon), values.data_ptr(), n, out.data_ptr(),
                               _stream_ptr(stream)))
    return out


def decompress(compressed: torch.Tensor, dtype, epsilon: float = DEFAULT_EPSILON, own_deltas: bool = False,
               out: Optional[torch.Tensor] = None, stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """Values from the int16 stream (decompress_1d, src/frsz.cc:132-150).
    own_deltas=False adds block 0's differences in every block, as the
    reference does; True adds each block's own (the inverse of compress)."""
    _require_cuda(compressed, "compressed")
    code = dtype_code(dtype)
    n = compressed.numel()
    tdt = torch.float32 if code == FRSZ2_FLOAT else torch.float64
    if out is None:
        out = torch.empty(n, dtype=tdt, device=compressed.device)
    check(lib().frsz1_decompress(code, float(epsilon), compressed.data_ptr(), n, out.data_ptr(),
                                 FRSZ1_OWN_DELTAS if own_deltas else 0, _stream_ptr(stream)))
    return out


class Frsz1Plugin:
    """The plugin's option surface ("frsz:epsilon", src/frsz.cc:20-47) over
    device tensors."""

    prefix = "frsz"

    def __init__(self, epsilon: float = DEFAULT_EPSILON):
        self.epsilon = float(epsilon)

    def get_options(self) -> dict:
        return {"frsz:epsilon": self.epsilon}

    def set_options(self, options: dict) -> int:
        if "frsz:epsilon" in options:
            self.epsilon = float(options["frsz:epsilon"])
        return 0

    def compress(self, values: torch.Tensor) -> torch.Tensor:
        return compress(values, self.epsilon)

    def decompress(self, compressed: torch.Tensor, dtype) -> torch.Tensor:
        return decompress(compressed, dtype, self.epsilon)
