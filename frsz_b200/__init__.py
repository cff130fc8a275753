"""frsz_b200 -- B200-native FRSZ2 fixed-rate floating-point compressor.

Byte-compatible with robertu94/frsz's ``frsz::frsz2_compressor`` (FRSZ2).
The codec runs as hand-written sm_100a CUDA kernels in libfrsz2_b200.so,
reached through the C ABI of include/frsz2_b200.h.  This package is the
Python host side: a mirror of the reference's compressor API and the
LibPressio-style ``frsz2`` plugin front end.
"""
from ._lib import FRSZ2_DOUBLE, FRSZ2_EDTYPE, FRSZ2_EFAIL, FRSZ2_FLOAT, FRSZ2_OK, Frsz2Error, lib
from .codec import (
    Frsz2Compressor,
    compress,
    compress_host,
    compressed_size,
    decompress,
    decompress_elements,
    decompress_elements_host,
    decompress_host,
    dispatch_frsz2_compression,
    dispatch_frsz2_decompression,
    exponent_size,
    word_bits,
)
from .plugin import Frsz2Plugin
from .batch import BatchArray, BatchPlan
from .krylov import CompressedBasis
from . import serve

__all__ = [
    "FRSZ2_DOUBLE", "FRSZ2_EDTYPE", "FRSZ2_EFAIL", "FRSZ2_FLOAT", "FRSZ2_OK", "Frsz2Error", "lib",
    "Frsz2Compressor", "compress", "compress_host", "compressed_size", "decompress", "decompress_elements",
    "decompress_elements_host", "decompress_host", "dispatch_frsz2_compression", "dispatch_frsz2_decompression", "exponent_size", "word_bits",
    "Frsz2Plugin", "BatchArray", "BatchPlan", "CompressedBasis",
]
