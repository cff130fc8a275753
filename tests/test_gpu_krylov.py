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


def edge_vector(n, E, seed):
    """Blocks whose exponents sit at the edges of the fused kernels' decode
    ranges (1002 / 1003 / 1023 at the top, -959 / -960 / -1000 at the
    bottom, 0), with zeros (zero codes), negative values and subnormals."""
    rng = np.random.default_rng(seed)
    x = np.empty(n, dtype=np.float64)
    exps = (1002, 1003, 1023, -959, -960, -1000, 0, 5, -3)
    for b in range(n // E):
        be = exps[(b + seed) % len(exps)]
        v = rng.uniform(-1.0, 1.0, E) * 2.0 ** be
        v[rng.integers(E)] = (1.0 + rng.random()) * 2.0 ** be * (1 if rng.random() < 0.5 else -1)
        v[rng.random(E) < 0.2] = 0.0
        if be <= -959:
            v[rng.random(E) < 0.1] = 5e-324 * rng.integers(1, 1000)
        x[b * E:(b + 1) * E] = v
    return x


@pytest.mark.parametrize("bits", [16, 21, 24, 32, 48])
def test_axpy_bit_exact_at_exponent_edges(cuda, bits):
    """y[i] = fma(c[j], V[j][i], y[i]) for j = 0 .. m-1, each rounded once:
    the fused axpy (which builds values of widths up to 32 bits without an
    integer-to-double conversion in the blocks whose exponent lies in
    [-959, 1002], and decodes the others as decompress does) equals that
    sequence bit for bit, computed here exactly with rationals."""
    from fractions import Fraction

    n, m, E = 2048, 3, 32
    basis = CompressedBasis(m, n, bits=bits, block_size=E)
    for j in range(m):
        basis.append(torch.from_numpy(edge_vector(n, E, 11 * j + bits)).cuda())
    V = torch.stack([basis.get(j) for j in range(m)]).cpu().numpy()
    rng = np.random.default_rng(bits)
    c = rng.uniform(0.25, 0.5, m) * np.where(rng.random(m) < 0.5, -1.0, 1.0)
    y0 = rng.standard_normal(n)
    y = torch.from_numpy(y0).cuda()
    basis.axpy(torch.from_numpy(c).cuda(), y)
    want = y0.copy()
    for j in range(m):
        cj = Fraction(float(c[j]))
        for i in range(n):
            want[i] = float(cj * Fraction(float(V[j, i])) + Fraction(float(want[i])))
    got = y.cpu().numpy()
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
