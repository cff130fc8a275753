"""Seeded synthetic inputs with the shapes and value distributions of the
FRSZ2 benchmark configurations (there is no public dataset for this codec).

numpy generators (``*_np``) are deterministic across machines with the same
numpy and feed the parity tests and golden fixtures; torch generators
(``*_cuda``) build the full-size arrays directly in HBM for the benchmark.
"""
from __future__ import annotations

import math

import numpy as np
import torch

# ---------------------------------------------------------------- numpy


def normal_np(n: int, dtype=np.float64, seed: int = 42) -> np.ndarray:
    """i.i.d. N(0, 1)."""
    return np.random.default_rng(seed).standard_normal(n).astype(dtype)


def reference_pattern(n: int, dtype=np.float64) -> np.ndarray:
    """The repeating values of the reference's end-to-end GPU test
    (test/test_frsz_gpu.cu:385-403)."""
    rep = np.array([1.0, 2.0, 3.0, 4.0, 0.25, -0.25, -0.125, 1 / 32.0, 0.125])
    return rep[np.arange(n) % rep.size].astype(dtype)


def loguniform_np(n: int, dtype=np.float64, seed: int = 42, lo: float = -30.0, hi: float = 30.0,
                  zero_frac: float = 0.01, subnormal_frac: float = 0.001) -> np.ndarray:
    """Random sign, magnitude 10^U(lo, hi), then `zero_frac` of the indices set
    to exact zero and `subnormal_frac` to subnormals uniform in (0, tiny)."""
    rng = np.random.default_rng(seed)
    x = np.where(rng.random(n) < 0.5, -1.0, 1.0) * np.power(10.0, rng.uniform(lo, hi, n))
    x = x.astype(dtype)
    tiny = np.finfo(dtype).tiny
    x[rng.random(n) < zero_frac] = 0
    sub = rng.random(n) < subnormal_frac
    x[sub] = (rng.random(int(sub.sum())) * float(tiny)).astype(dtype)
    return x


def loguniform_host(n: int, dtype=np.float64, seed: int = 42, chunk: int = 1 << 22, threads: int = 0,
                    **kw) -> np.ndarray:
    """loguniform_np's distribution for large n, generated on the host in
    chunks of `chunk` values, chunk c from its own generator seeded with
    (seed, c), on `threads` threads (0: all host cores).  The values depend
    only on (n, dtype, seed, chunk), not on the thread count, so a GPU run
    and a CPU run that both call this get the same array."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    out = np.empty(n, dtype=dtype)

    def fill(c):
        s = c * chunk
        m = min(chunk, n - s)
        out[s:s + m] = loguniform_np(m, dtype, seed=[seed, c], **kw)

    with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as ex:
        list(ex.map(fill, range(-(-n // chunk))))
    return out


def uniform_np(n: int, lo: float, hi: float, dtype=np.float32, seed: int = 42) -> np.ndarray:
    return np.random.default_rng(seed).uniform(lo, hi, n).astype(dtype)


# ---------------------------------------------------------------- torch / CUDA


def normal_cuda(n: int, dtype=torch.float64, seed: int = 42, device="cuda") -> torch.Tensor:
    g = torch.Generator(device=device).manual_seed(seed)
    return torch.randn(n, generator=g, device=device, dtype=dtype)


def loguniform_cuda(n: int, dtype=torch.float64, seed: int = 42, lo: float = -30.0, hi: float = 30.0,
                    zero_frac: float = 0.01, subnormal_frac: float = 0.001, device="cuda",
                    chunk: int = 1 << 26) -> torch.Tensor:
    """Device version of loguniform_np, generated in chunks to bound temporaries."""
    g = torch.Generator(device=device).manual_seed(seed)
    out = torch.empty(n, dtype=dtype, device=device)
    tiny = torch.finfo(dtype).tiny
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        u = torch.rand(m, generator=g, device=device, dtype=torch.float64)
        sign = torch.where(torch.rand(m, generator=g, device=device) < 0.5, -1.0, 1.0).to(torch.float64)
        x = sign * torch.pow(10.0, lo + (hi - lo) * u)
        r = torch.rand(m, generator=g, device=device)
        x = torch.where(r < zero_frac, torch.zeros_like(x), x)
        sub = (r >= zero_frac) & (r < zero_frac + subnormal_frac)
        x = torch.where(sub, torch.rand(m, generator=g, device=device, dtype=torch.float64) * tiny, x)
        out[s:s + m] = x.to(dtype)
    return out


def sinusoid_field_cuda(nx: int = 512, ny: int = 512, nz: int = 512, seed: int = 42, waves: int = 8,
                        lmin: float = 8.0, lmax: float = 256.0, noise: float = 1e-3, dtype=torch.float32,
                        device="cuda") -> torch.Tensor:
    """3-D field: sum of `waves` plane sinusoids with wavelengths log-spaced in
    [lmin, lmax] cells, random unit directions and phases, plus N(0, noise^2).
    Built slab by slab along z; returns a flat (nz*ny*nx) tensor, x fastest."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    lam = torch.exp(torch.linspace(math.log(lmin), math.log(lmax), waves, dtype=torch.float64))
    d = torch.randn(waves, 3, generator=g, dtype=torch.float64)
    d = d / d.norm(dim=1, keepdim=True)
    phase = torch.rand(waves, generator=g, dtype=torch.float64) * 2 * math.pi
    k = (2 * math.pi / lam)[:, None] * d  # (waves, 3)
    gd = torch.Generator(device=device).manual_seed(seed + 1)
    out = torch.empty(nz * ny * nx, dtype=dtype, device=device)
    xs = torch.arange(nx, device=device, dtype=torch.float32)
    ys = torch.arange(ny, device=device, dtype=torch.float32)
    plane = nx * ny
    for z in range(nz):
        acc = torch.zeros(ny, nx, device=device, dtype=torch.float32)
        for w in range(waves):
            kx, ky, kz = (float(v) for v in k[w])
            acc += torch.sin(kx * xs[None, :] + ky * ys[:, None] + (kz * z + float(phase[w])))
        acc += noise * torch.randn(ny, nx, generator=gd, device=device, dtype=torch.float32)
        out[z * plane:(z + 1) * plane] = acc.reshape(-1).to(dtype)
    return out
