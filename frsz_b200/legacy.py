"""The reference's legacy "frsz" codec (the LibPressio plugin "frsz",
src/frsz.cc:15-165) on the GPU: epsilon quantization, int16 differences
within blocks of 256 values.  compress / decompress take device tensors;
Frsz1Plugin is the plugin's front end over host or device arrays.  The work
runs in the library's CUDA kernels (frsz_b200/csrc/frsz1_legacy.cu)."""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from ._lib import FRSZ2_EFAIL, FRSZ2_FLOAT, Frsz2Error, check, lib
from .codec import _require_cuda, _stream_ptr, dtype_code

FRSZ1_OWN_DELTAS = 1
DEFAULT_EPSILON = 1e-4  # "frsz:epsilon" (src/frsz.cc:160)


def compress(values: torch.Tensor, epsilon: float = DEFAULT_EPSILON, out: Optional[torch.Tensor] = None,
             stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """int16 stream of a CUDA float32 / float64 tensor (compress_1d,
    src/frsz.cc:103-130)."""
    _require_cuda(values, "values")
    n = values.numel()
    if out is None:
        out = torch.empty(n, dtype=torch.int16, device=values.device)
    else:
        _require_cuda(out, "out")
        if out.dtype != torch.int16 or out.numel() < n:
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
    else:
        _require_cuda(out, "out")
        if out.dtype != tdt or out.numel() < n:
            raise Frsz2Error(FRSZ2_EFAIL, f"out must be a {tdt} tensor of at least n elements")
    check(lib().frsz1_decompress(code, float(epsilon), compressed.data_ptr(), n, out.data_ptr(),
                                 FRSZ1_OWN_DELTAS if own_deltas else 0, _stream_ptr(stream)))
    return out


def legacy_length(shape) -> int:
    """How many values the plugin codes for an array of this shape: the
    reference takes normalized_dims(1).at(0) (src/frsz.cc:108, 139), and
    LibPressio's pressio_data::normalized_dims drops the dimensions of extent
    1 and cuts the list to its first entry, filling 0 when none is left.  So a
    1-D array codes all its values, a 2-D array only its first extent, and a
    single value none."""
    dims = [int(d) for d in shape if int(d) > 1]
    return dims[0] if dims else 0


class Frsz1Plugin:
    """The LibPressio "frsz" compressor plugin front end (src/frsz.cc:17-161):
    option "frsz:epsilon" (default 1e-4), configuration and documentation
    entries, version 0.0.6 (the project version, CMakeLists.txt:3), prefix
    "frsz", status 1 with the reference's message for other dtypes.  Inputs
    are numpy arrays (host) or torch CUDA tensors (device); compress returns
    the int16 stream as bytes (2 per coded value) in the same place.  The
    work runs in the library's CUDA kernels either way: host arrays are
    copied to the current device and back.  A status 2 carries the library's
    message (a device failure, or epsilon <= 0, which the library rejects)."""

    prefix = "frsz"

    def __init__(self, epsilon: float = DEFAULT_EPSILON):
        self.epsilon = float(epsilon)
        self.error_code = 0
        self.error_msg = ""

    # ---- options (src/frsz.cc:19-46)
    def get_options(self) -> dict:
        return {"frsz:epsilon": self.epsilon}

    def set_options(self, options: dict) -> int:
        if "frsz:epsilon" in options:
            self.epsilon = float(options["frsz:epsilon"])
        return 0

    def get_configuration(self) -> dict:
        return {"pressio:thread_safe": "multiple", "pressio:stability": "experimental"}

    def get_documentation(self) -> dict:
        return {
            "pressio:description": "a fixed rate version of the SZ Algorithm",
            "frsz:epsilon": "\"absolute error bound\" applied during quantization; because frsz does not store "
                            "unpredictable values, this is not a true absolute error bound",
        }

    def version(self) -> str:
        return "0.0.6"

    def major_version(self) -> int:
        return 0

    def minor_version(self) -> int:
        return 0

    def patch_version(self) -> int:
        return 6

    def get_metrics_results(self) -> dict:
        return {}

    # ---- errors (src/frsz.cc:57-58, 74-75)
    def _set_error(self, code: int, msg: str) -> int:
        self.error_code, self.error_msg = code, msg
        return code

    def _dtype(self, dtype):
        try:
            return dtype_code(dtype)
        except Frsz2Error:
            return None

    # ---- codec (src/frsz.cc:48-80, 105-158)
    def compress(self, data):
        """Returns (status, bytes): the int16 stream of the first
        legacy_length(shape) values, as uint8 (a CUDA tensor for a CUDA
        input, else a numpy array)."""
        if self._dtype(data.dtype) is None:
            return self._set_error(1, "unsupported type: currently only floating point supported"), None
        n = legacy_length(data.shape)
        try:
            if isinstance(data, torch.Tensor):
                q = compress(data.reshape(-1)[:n], self.epsilon)
                return 0, q.view(torch.uint8)
            flat = np.ascontiguousarray(data).reshape(-1)[:n]
            if n == 0:
                return 0, np.zeros(0, dtype=np.uint8)
            q = compress(torch.from_numpy(flat).cuda(), self.epsilon)
            return 0, q.cpu().numpy().view(np.uint8)
        except Frsz2Error as e:
            return self._set_error(2, str(e)), None

    def decompress(self, compressed, output) -> int:
        """Fills the first legacy_length(output.shape) values of `output`
        (whose dtype and shape the caller chose) from the int16 stream
        `compressed` (bytes or int16, host or device), adding block 0's
        differences in every block as the reference does."""
        code = self._dtype(output.dtype)
        if code is None:
            return self._set_error(1, "unsupported type: currently only floating point supported")
        n = legacy_length(output.shape)
        try:
            if isinstance(compressed, torch.Tensor):
                b = compressed.reshape(-1).view(torch.uint8)
                q = b[: b.numel() // 2 * 2].view(torch.int16)
            else:
                b = np.ascontiguousarray(compressed).reshape(-1).view(np.uint8)
                q = torch.from_numpy(b[: b.size // 2 * 2].view(np.int16))
            if q.numel() < n:
                return self._set_error(2, "compressed input is shorter than the format requires")
            if n == 0:
                return 0
            q = q[:n]
            if isinstance(output, torch.Tensor):
                _require_cuda(output, "output")
                flat = output.view(-1)[:n]
                decompress(q.to(output.device), output.dtype, self.epsilon, out=flat)
            else:
                if not output.flags.c_contiguous:
                    raise Frsz2Error(FRSZ2_EFAIL, "output must be contiguous")
                output.reshape(-1)[:n] = decompress(q.cuda(), output.dtype, self.epsilon).cpu().numpy()
        except Frsz2Error as e:
            return self._set_error(2, str(e))
        return 0

    def clone(self) -> "Frsz1Plugin":
        return Frsz1Plugin(self.epsilon)
