"""Host-side logic of bench.py (no GPU): workload names, algorithmic bytes."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_named_and_generic_workloads():
    assert bench.workload_spec("loguniform_f64_2p28_b21_e32") == ("loguniform", "float64", 1 << 28, 21, 32)
    assert bench.workload_spec("normal_f32_2p26_b28_e8") == ("normal", "float32", 1 << 26, 28, 8)
    assert bench.workload_spec("normal_f64_2p27_b32_e100") == ("normal", "float64", 1 << 27, 32, 100)
    # the named table wins for the view workloads, which carry an offset
    assert bench.workload_spec("normal_f32_2p28_b16_e32_off1")[5] == 1


@pytest.mark.parametrize("name", ["normal_f32_2p28_b33_e32",   # above fp32's 32 bits
                                  "normal_f64_2p28_b3_e32",    # below 4 bits
                                  "uniform_f32_2p20_b16_e32",  # unknown kind
                                  "normal_f32_2p40_b16_e32",   # too large
                                  "normal_f32_2p20_b16_e0"])   # no block size
def test_rejected_workloads(name):
    with pytest.raises(SystemExit):
        bench.workload_spec(name)


def test_algorithmic_bytes_match_the_layout():
    # values + per block (words + one exponent); the 256-byte pad is not counted
    n, E = 1 << 20, 32
    assert bench.algorithmic_bytes("float64", n, 32, E) == n * 8 + (n // E) * (E * 4 + 4)
    # 21 bits in 32-bit words: 672 bits per block of 32 = 21 words
    assert bench.algorithmic_bytes("float64", n, 21, E) == n * 8 + (n // E) * (21 * 4 + 4)
    # padded blocks: 24 values at 21 bits = 504 bits -> 16 words
    assert bench.algorithmic_bytes("float32", 48, 21, 24) == 48 * 4 + 2 * (16 * 4 + 4)
    # 8-bit words and exponents
    assert bench.algorithmic_bytes("float32", 100, 5, 8) == 100 * 4 + 13 * (5 + 1)
