"""GPU: dot / axpy fused with decompression over a compressed fp64 basis,
against torch fp64 on the decompressed vectors.  Tolerance: the fused sums
differ from torch's only in summation order, so |got - want| <= 1e-12 *
sum(|terms|) (with n, m here the order error is below 1e-14)."""
import numpy as np
import pytest
import torch

import frsz_b200
from frsz_b200 import CompressedBasis, workloads

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("bits,E,n,m", [(32, 32, 100_003, 20), (21, 32, 65_536, 7), (16, 64, 10_001, 33),
                                        (64, 16, 5_000, 3), (24, 32, 777, 1),
                                        # code stream ending off a 16-byte boundary
                                        (21, 32, 100_003, 5), (48, 4, 70_001, 4),
                                        # exponent blocks longer than a slice of the dot
                                        (16, 4096, 300_001, 3), (32, 65536, 200_000, 2)])
def test_dot_and_axpy(cuda, bits, E, n, m):
    basis = CompressedBasis(m, n, bits=bits, block_size=E)
    g = torch.Generator(device="cuda").manual_seed(bits + m)
    for j in range(m):
        basis.append(torch.randn(n, generator=g, device="cuda", dtype=torch.float64) * 10.0 ** (j % 5 - 2))
    V = torch.stack([basis.get(j) for j in range(m)])
    w = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    h = basis.dot(w)
    want = V @ w
    scale = V.abs() @ w.abs()
    assert torch.all((h - want).abs() <= TOL * scale + 1e-300)
    h2 = basis.dot(w)  # the workspace is reused; the result is the same bits
    assert torch.equal(h, h2)
    c = torch.randn(m, generator=g, device="cuda", dtype=torch.float64)
    y = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    y0 = y.clone()
    basis.axpy(c, y)
    want_y = y0 + c @ V
    scale_y = y0.abs() + c.abs() @ V.abs()
    assert torch.all((y - want_y).abs() <= TOL * scale_y)


def test_partial_basis_and_errors(cuda):
    basis = CompressedBasis(4, 3000, bits=32)
    for j in range(4):
        basis.append(torch.full((3000,), float(j + 1), device="cuda", dtype=torch.float64))
    w = torch.ones(3000, device="cuda", dtype=torch.float64)
    assert torch.equal(basis.dot(w, m=2).cpu(), torch.tensor([3000.0, 6000.0], dtype=torch.float64))
    bad = CompressedBasis(1, 100, bits=17)
    bad.append(torch.ones(100, device="cuda", dtype=torch.float64))
    with pytest.raises(frsz_b200.Frsz2Error, match="no instance for 17 bits"):
        bad.dot(torch.ones(100, device="cuda", dtype=torch.float64))


def test_dot_with_w_not_32_byte_aligned(cuda):
    """w as a view at an 8-byte offset: the dot reads it with scalar loads."""
    n, m = 50_001, 6
    basis = CompressedBasis(m, n, bits=32, block_size=32)
    g = torch.Generator(device="cuda").manual_seed(7)
    for j in range(m):
        basis.append(torch.randn(n, generator=g, device="cuda", dtype=torch.float64))
    V = torch.stack([basis.get(j) for j in range(m)])
    wbig = torch.randn(n + 1, generator=g, device="cuda", dtype=torch.float64)
    w = wbig[1:]
    assert w.data_ptr() % 32 != 0
    h = basis.dot(w)
    assert torch.all((h - V @ w).abs() <= TOL * (V.abs() @ w.abs()) + 1e-300)
