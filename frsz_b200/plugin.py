"""The reference's LibPressio ``frsz2`` compressor plugin front end
(robertu94/frsz src/frsz2.cc:25-208) over the B200 codec.

Same option keys and defaults (``frsz2:bits`` = 32, ``frsz2:max_exp_block_size``
= 32), supported values (float bits 4..32, double bits 4..64, block sizes
2..1024 powers of two), configuration / documentation entries, version
0.0.2, prefix ``frsz2`` and error behaviour: status 1 "unsupported dtype",
status 2 with the dispatch's message.  Inputs are numpy arrays (host) or
torch CUDA tensors (device); compress returns a buffer in the same place.

Compress sizes its output with compute_compressed_memory_size_byte; the
reference's output_size() (src/frsz2.cc:136-150) is smaller than what its
codec writes.
"""
from __future__ import annotations

from typing import Any, Dict, Tuple

import numpy as np
import torch

from ._lib import Frsz2Error
from . import codec

_SUPPORTED_E = (2, 4, 8, 16, 32, 64, 128, 256, 512, 1024)


class Frsz2Plugin:
    prefix = "frsz2"

    def __init__(self):
        self.bits = 32
        self.max_exp_block_size = 32
        self.error_code = 0
        self.error_msg = ""

    # ---- options (src/frsz2.cc:28-35, 58-64)
    def get_options(self) -> Dict[str, int]:
        return {"frsz2:bits": self.bits, "frsz2:max_exp_block_size": self.max_exp_block_size}

    def set_options(self, options: Dict[str, Any]) -> int:
        if "frsz2:bits" in options:
            self.bits = int(options["frsz2:bits"])
        if "frsz2:max_exp_block_size" in options:
            self.max_exp_block_size = int(options["frsz2:max_exp_block_size"])
        return 0

    def get_configuration(self) -> Dict[str, str]:
        return {"pressio:thread_safe": "multiple", "pressio:stability": "experimental"}

    def get_documentation(self) -> Dict[str, str]:
        return {
            "pressio:description": "a fixed rate compressor which uses block exponents + rounding",
            "frsz2:bits": "the number of bits to use per symbol",
            "frsz2:max_exp_block_size": "the number of elements to have a common exponent. Supported values: "
                                        "2, 4, 8, 16, 32, 64, 128, 256, 512, 1024",
        }

    def version(self) -> str:
        return "0.0.2"

    def major_version(self) -> int:
        return 0

    def minor_version(self) -> int:
        return 0

    def patch_version(self) -> int:
        return 2

    # ---- errors
    def _set_error(self, code: int, msg: str) -> int:
        self.error_code, self.error_msg = code, msg
        return code

    def _check(self, dtype) -> int:
        try:
            code = codec.dtype_code(dtype)
        except Frsz2Error:
            return self._set_error(1, "unsupported dtype")
        max_bits = 32 if code == 0 else 64
        if not 4 <= self.bits <= max_bits:
            return self._set_error(2, f"Unsupported number of bits: {self.bits}")
        if self.max_exp_block_size not in _SUPPORTED_E:
            return self._set_error(2, f"Unsupported exponent block size: {self.max_exp_block_size}")
        return 0

    # ---- codec (src/frsz2.cc:152-186)
    def compress(self, data) -> Tuple[int, Any]:
        """Returns (status, compressed buffer)."""
        rc = self._check(data.dtype)
        if rc:
            return rc, None
        try:
            if isinstance(data, torch.Tensor):
                return 0, codec.compress(data.reshape(-1), self.bits, self.max_exp_block_size)
            return 0, codec.compress_host(np.ascontiguousarray(data).reshape(-1), self.bits,
                                          self.max_exp_block_size)
        except Frsz2Error as e:
            return self._set_error(2, str(e)), None

    def decompress(self, compressed, output) -> int:
        """Fills `output`, whose dtype and shape the caller chose."""
        rc = self._check(output.dtype)
        if rc:
            return rc
        n = int(np.prod(output.shape)) if len(output.shape) else 1
        try:
            if isinstance(output, torch.Tensor):
                flat = output.view(-1)
                codec.decompress(compressed, n, output.dtype, self.bits, self.max_exp_block_size, out=flat)
            else:
                flat = output.reshape(-1)
                codec.decompress_host(compressed, n, output.dtype, self.bits, self.max_exp_block_size, out=flat)
                if not np.shares_memory(flat, output):
                    output[...] = flat.reshape(output.shape)
        except Frsz2Error as e:
            return self._set_error(2, str(e))
        return 0

    def clone(self) -> "Frsz2Plugin":
        p = Frsz2Plugin()
        p.set_options(self.get_options())
        return p
