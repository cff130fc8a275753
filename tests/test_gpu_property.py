"""GPU: property-based parity -- random float types, widths, block sizes,
sizes and values (NaN, +-Inf, +-0, subnormals included) through the C ABI,
against the oracle, whole canary buffers and decoded bit patterns."""
import numpy as np
import pytest
import torch
from hypothesis import HealthCheck, given, settings, strategies as st

import oracle
import frsz_b200

pytestmark = pytest.mark.gpu


@st.composite
def gpu_case(draw):
    is64 = draw(st.booleans())
    dtype = np.float64 if is64 else np.float32
    bits = draw(st.integers(4, 64 if is64 else 32))
    E = draw(st.sampled_from([1, 2, 3, 4, 8, 16, 32, 64, 128, 256, 1024]))
    n = draw(st.integers(0, 9000))
    seed = draw(st.integers(0, 2 ** 31))
    rng = np.random.default_rng(seed)
    lo, hi = (-35, 35) if not is64 else ((-30, 30) if bits <= 8 else (-300, 300))
    x = (np.where(rng.random(n) < 0.5, -1.0, 1.0) * 10.0 ** rng.uniform(lo, hi, n)).astype(dtype)
    k = draw(st.integers(0, 8))
    specials = np.array([np.nan, np.inf, -np.inf, 0.0, -0.0, np.finfo(dtype).smallest_subnormal], dtype=dtype)
    if n:
        x[rng.integers(0, n, k)] = specials[rng.integers(0, specials.size, k)]
    return x, bits, E


@settings(max_examples=120, deadline=None, suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])
@given(gpu_case())
def test_property_kernels_equal_oracle(cuda, case):
    x, bits, E = case
    size = frsz_b200.compressed_size(x.dtype, bits, E, x.size)
    buf = torch.full((size,), 0xC7, dtype=torch.uint8, device="cuda")
    if x.size:
        frsz_b200.compress(torch.from_numpy(x).cuda(), bits, E, out=buf)
    ref = oracle.compress(x, bits, E, canary=0xC7)
    assert np.array_equal(buf.cpu().numpy(), ref)
    if x.size:
        y = frsz_b200.decompress(torch.from_numpy(ref).cuda(), x.size, x.dtype, bits, E).cpu().numpy()
        assert np.array_equal(y.view(np.uint8), oracle.decompress(ref, x.size, x.dtype, bits, E).view(np.uint8))
