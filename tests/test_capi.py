"""CPU: the C-ABI library loads, exports every symbol include/*.h declares,
and its host logic (size algebra, argument checks, error messages) matches
the reference -- no kernel is launched here."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import oracle
import frsz_b200
from frsz_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "sizeof", "defined"):
                names.add(name)
    return names


def test_header_symbols_exported():
    lib = frsz_b200.lib()
    names = declared_functions()
    assert {"register_frsz", "frsz2_compress", "frsz2_decompress", "frsz2_compressed_size"} <= names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_functions() <= set(_lib.SIGNATURES)


def test_register_frsz_is_callable():
    frsz_b200.lib().register_frsz()
    assert frsz_b200.lib().frsz2_version().decode().startswith("0.0.2")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_sizes_match_oracle(dtype):
    max_bits = 32 if dtype == np.float32 else 64
    for bits in range(4, max_bits + 1):
        for E in (1, 2, 3, 4, 5, 8, 32, 64, 1000, 1024, 4096):
            for n in (0, 1, 31, 32, 33, 4097, 1 << 28):
                assert frsz_b200.compressed_size(dtype, bits, E, n) == oracle.compressed_bytes(bits, E, n)
                assert frsz_b200.exponent_size(dtype, bits, E, n) == oracle.exponent_bytes(bits, E, n)


def test_error_codes_and_messages():
    """Status 1 for a dtype the plugin rejects, 2 with the reference's
    runtime_error text for unsupported bits / block sizes
    (src/frsz2.cc:164-168, include/frsz2.hpp:1300, 1326)."""
    lib = frsz_b200.lib()
    out = ctypes.c_uint64()
    assert lib.frsz2_compressed_size(7, 16, 32, 10, ctypes.byref(out)) == 1
    assert lib.frsz2_last_error() == b"unsupported dtype"
    assert lib.frsz2_compressed_size(0, 33, 32, 10, ctypes.byref(out)) == 2
    assert lib.frsz2_last_error() == b"Unsupported number of bits: 33"
    assert lib.frsz2_compressed_size(1, 3, 32, 10, ctypes.byref(out)) == 2
    assert lib.frsz2_last_error() == b"Unsupported number of bits: 3"
    assert lib.frsz2_compressed_size(1, 16, 0, 10, ctypes.byref(out)) == 2
    assert lib.frsz2_last_error() == b"Unsupported exponent block size: 0"
    with pytest.raises(frsz_b200.Frsz2Error) as ei:
        frsz_b200.compressed_size(np.int32, 16, 32, 10)
    assert ei.value.code == 1
    # bad arguments are rejected before any device work
    assert lib.frsz2_compress(0, 64, 32, None, 10, None, None) == 2
    assert lib.frsz2_compress(0, 16, 32, None, 10, None, None) == 2
    assert lib.frsz2_last_error() == b"null pointer"
    assert lib.frsz2_compress(0, 16, 32, None, 0, None, None) == 0  # n == 0 is a no-op


def test_dispatch_rejects_unlisted_values():
    with pytest.raises(frsz_b200.Frsz2Error, match="Unsupported number of bits: 7"):
        frsz_b200.dispatch_frsz2_compression(np.float32, [8, 16, 32], 7, [32], 32, np.zeros(4, np.float32), 4,
                                             np.zeros(300, np.uint8))
    with pytest.raises(frsz_b200.Frsz2Error, match="Unsupported exponent block size: 48"):
        frsz_b200.dispatch_frsz2_compression(np.float32, [16], 16, [32, 64], 48, np.zeros(4, np.float32), 4,
                                             np.zeros(300, np.uint8))


def test_compressor_view_geometry():
    c = frsz_b200.Frsz2Compressor(21, 32, np.float64, np.zeros(oracle.compressed_bytes(21, 32, 100), np.uint8), 100)
    assert c.uint_compressed_size_bit == 32
    assert c.compressed_block_size_element_count == 21
    assert c.compressed_block_size_byte == 84
    assert c.compute_exponent_block_size_byte(100) == 4 * 4 + 240
    assert c.get_exponent_data().dtype == np.int32 and c.get_exponent_data().size == 4
    with pytest.raises(frsz_b200.Frsz2Error):
        frsz_b200.Frsz2Compressor(40, 32, np.float32, None, 0)
