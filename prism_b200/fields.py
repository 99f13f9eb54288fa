"""Seeded synthetic scientific fields used by the tests, the golden-fixture
script and the benchmark.

All fields are C-ordered numpy arrays ``a[z][y][x]`` (x fastest), i.e. the raw
little-endian layout the PRISM CLI reads with ``-3 nx ny nz``.  The generators
stand in for the datasets the reference's README names (SDRBench Miranda etc.),
which are not available offline; they reproduce the shapes, dtypes and value
distributions of the benchmark configurations.

* ``sinusoid``   - sum of 8 random plane waves + N(0, 1e-3) noise (smooth).
* ``grf``        - Gaussian random field with an isotropic k^-5/3 power
                   spectrum (inverse rFFT of seeded complex normals), mapped
                   affinely to [lo, hi].
* ``voronoi``    - piecewise-smooth field: nearest-of-64-seeds cells, each a
                   random quadratic polynomial, 30% of cells exactly 0.0, plus
                   0.1% isolated spikes of +-1e3 (sparse/sharp).
"""
from __future__ import annotations

import numpy as np


def sinusoid(shape, dtype=np.float32, seed=0, waves=8, noise=1e-3):
    """Sum of ``waves`` sinusoids with integer wavenumbers 1..8 per axis."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.1, 1.0, waves)
    phase = rng.uniform(0.0, 2 * np.pi, waves)
    k = rng.integers(1, 9, size=(waves, 3))
    z = np.arange(nz, dtype=np.float64)[:, None, None] / max(nz, 1)
    y = np.arange(ny, dtype=np.float64)[None, :, None] / max(ny, 1)
    x = np.arange(nx, dtype=np.float64)[None, None, :] / max(nx, 1)
    out = np.zeros(shape, dtype=np.float64)
    for i in range(waves):
        out += amp[i] * np.sin(2 * np.pi * (k[i, 0] * x + k[i, 1] * y + k[i, 2] * z) + phase[i])
    out += rng.normal(0.0, noise, size=shape)
    return out.astype(dtype)


def grf(shape, dtype=np.float64, seed=1, slope=-5.0 / 3.0, lo=0.9, hi=3.0):
    """Isotropic Gaussian random field with power spectrum P(k) ~ k^slope."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    kz = np.fft.fftfreq(nz)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    kx = np.fft.rfftfreq(nx)[None, None, :]
    kk = np.sqrt(kz * kz + ky * ky + kx * kx)
    kk[0, 0, 0] = 1.0
    amp = kk ** (slope / 2.0)
    amp[0, 0, 0] = 0.0
    spec = (rng.standard_normal(amp.shape) + 1j * rng.standard_normal(amp.shape)) * amp
    f = np.fft.irfftn(spec, s=shape, axes=(0, 1, 2))
    fmin, fmax = f.min(), f.max()
    f = lo + (hi - lo) * (f - fmin) / (fmax - fmin)
    return f.astype(dtype)


def voronoi(shape, dtype=np.float32, seed=2, cells=64, zero_frac=0.3,
            spike_frac=1e-3, spike_amp=1e3, slab=16):
    """Piecewise-quadratic Voronoi field with zero cells and isolated spikes."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    seeds = rng.uniform(0.0, 1.0, size=(cells, 3)) * np.array([nz, ny, nx])
    coef = rng.normal(0.0, 1.0, size=(cells, 10))
    zero = rng.uniform(0.0, 1.0, cells) < zero_frac
    coef[zero] = 0.0
    out = np.empty(shape, dtype=dtype)
    y = (np.arange(ny, dtype=np.float32) / ny)[None, :, None]
    x = (np.arange(nx, dtype=np.float32) / nx)[None, None, :]
    sy = np.arange(ny, dtype=np.float32)[None, :, None]
    sx = np.arange(nx, dtype=np.float32)[None, None, :]
    for z0 in range(0, nz, slab):
        z1 = min(nz, z0 + slab)
        sz = np.arange(z0, z1, dtype=np.float32)[:, None, None]
        best = np.full((z1 - z0, ny, nx), np.inf, dtype=np.float32)
        owner = np.zeros((z1 - z0, ny, nx), dtype=np.int16)
        for c in range(cells):
            d = (sz - seeds[c, 0]) ** 2 + (sy - seeds[c, 1]) ** 2 + (sx - seeds[c, 2]) ** 2
            m = d < best
            best = np.where(m, d, best)
            owner = np.where(m, np.int16(c), owner)
        zz = (sz / nz)
        cc = coef[owner]
        v = (cc[..., 0] + cc[..., 1] * x + cc[..., 2] * y + cc[..., 3] * zz
             + cc[..., 4] * x * x + cc[..., 5] * y * y + cc[..., 6] * zz * zz
             + cc[..., 7] * x * y + cc[..., 8] * y * zz + cc[..., 9] * x * zz)
        out[z0:z1] = v.astype(dtype)
    n = out.size
    nspk = int(round(n * spike_frac))
    if nspk:
        idx = rng.choice(n, size=nspk, replace=False)
        sign = np.where(rng.uniform(0.0, 1.0, nspk) < 0.5, -1.0, 1.0)
        out.reshape(-1)[idx] = (sign * spike_amp).astype(dtype)
    return out


GENERATORS = {"sinusoid": sinusoid, "grf": grf, "voronoi": voronoi}


def make(kind, shape, dtype, seed):
    """Dispatch by generator name; ``shape`` is (nz, ny, nx)."""
    return GENERATORS[kind](tuple(shape), dtype=np.dtype(dtype), seed=seed)


# ---- device-side generators (torch, for benchmark-scale inputs) -------------
# Same families as above, generated on the GPU so that multi-GB inputs take
# seconds; the values differ from the numpy versions (different RNG streams).

def device_sinusoid(shape, dtype, seed, device="cuda", waves=8, noise=1e-3):
    import torch
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.1, 1.0, waves)
    phase = rng.uniform(0.0, 2 * np.pi, waves)
    k = rng.integers(1, 9, size=(waves, 3))
    z = torch.arange(nz, device=device, dtype=torch.float64)[:, None, None] / max(nz, 1)
    y = torch.arange(ny, device=device, dtype=torch.float64)[None, :, None] / max(ny, 1)
    x = torch.arange(nx, device=device, dtype=torch.float64)[None, None, :] / max(nx, 1)
    out = torch.zeros(shape, device=device, dtype=torch.float64)
    for i in range(waves):
        out += float(amp[i]) * torch.sin(2 * np.pi * (int(k[i, 0]) * x + int(k[i, 1]) * y + int(k[i, 2]) * z)
                                         + float(phase[i]))
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    out += noise * torch.randn(shape, device=device, dtype=torch.float64, generator=g)
    return out.to(torch.float32 if np.dtype(dtype) == np.float32 else torch.float64)


def device_grf(shape, dtype, seed, device="cuda", slope=-5.0 / 3.0, lo=0.9, hi=3.0):
    import torch
    nz, ny, nx = shape
    kz = torch.fft.fftfreq(nz, device=device, dtype=torch.float32)[:, None, None]
    ky = torch.fft.fftfreq(ny, device=device, dtype=torch.float32)[None, :, None]
    kx = torch.fft.rfftfreq(nx, device=device, dtype=torch.float32)[None, None, :]
    kk = torch.sqrt(kz * kz + ky * ky + kx * kx)
    kk[0, 0, 0] = 1.0
    amp = kk ** (slope / 2.0)
    amp[0, 0, 0] = 0.0
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    spec = torch.complex(torch.randn(amp.shape, device=device, generator=g),
                         torch.randn(amp.shape, device=device, generator=g)) * amp
    del kk, amp
    f = torch.fft.irfftn(spec, s=shape, dim=(0, 1, 2))
    del spec
    fmin, fmax = f.min(), f.max()
    f = lo + (hi - lo) * (f - fmin) / (fmax - fmin)
    return f.to(torch.float32 if np.dtype(dtype) == np.float32 else torch.float64)


def uneven_mix(count=64, seed=47, lo=32, hi=2048, cap3=512 ** 3):
    """The uneven batch: `count` fields, dimensionality uniform on {1, 2, 3},
    per-axis extents log-uniform in [lo, hi], 3-D volumes capped at `cap3`
    values (axes scaled down together), alternating smooth sinusoid sums and
    k^-5/3 random fields.  Returns [(kind, (nx, ny, nz))].  The default seed
    draws 5.96 GB of float32 in total (most draws give 3-4 GB; the batch is
    specified at about 6 GB)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        d = int(rng.integers(1, 4))
        ext = np.exp(rng.uniform(np.log(lo), np.log(hi), d))
        if d == 3 and np.prod(ext) > cap3:
            ext = ext * (cap3 / np.prod(ext)) ** (1.0 / 3.0)
        e = [max(lo, int(v)) for v in ext] + [1] * (3 - d)
        out.append(("sinusoid" if i % 2 == 0 else "grf", (e[0], e[1], e[2])))
    return out


def device_voronoi(shape, dtype, seed, device="cuda", cells=64, zero_frac=0.3, spike_frac=1e-3, spike_amp=1e3,
                   slab=16):
    """Device version of `voronoi` (same construction, torch RNG)."""
    import torch
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    seeds = torch.tensor(rng.uniform(0.0, 1.0, size=(cells, 3)) * np.array([nz, ny, nx]), device=device,
                         dtype=torch.float32)
    coef = rng.normal(0.0, 1.0, size=(cells, 10))
    coef[rng.uniform(0.0, 1.0, cells) < zero_frac] = 0.0
    coef = torch.tensor(coef, device=device, dtype=torch.float32)
    tdt = torch.float32 if np.dtype(dtype) == np.float32 else torch.float64
    out = torch.empty(shape, device=device, dtype=tdt)
    y = (torch.arange(ny, device=device, dtype=torch.float32) / ny)[None, :, None]
    x = (torch.arange(nx, device=device, dtype=torch.float32) / nx)[None, None, :]
    sy = torch.arange(ny, device=device, dtype=torch.float32)[None, :, None]
    sx = torch.arange(nx, device=device, dtype=torch.float32)[None, None, :]
    for z0 in range(0, nz, slab):
        z1 = min(nz, z0 + slab)
        sz = torch.arange(z0, z1, device=device, dtype=torch.float32)[:, None, None]
        best = torch.full((z1 - z0, ny, nx), float("inf"), device=device)
        owner = torch.zeros((z1 - z0, ny, nx), device=device, dtype=torch.long)
        for c in range(cells):
            d = (sz - seeds[c, 0]) ** 2 + (sy - seeds[c, 1]) ** 2 + (sx - seeds[c, 2]) ** 2
            m = d < best
            best = torch.where(m, d, best)
            owner = torch.where(m, torch.full_like(owner, c), owner)
        zz = sz / nz
        cc = coef[owner]
        v = (cc[..., 0] + cc[..., 1] * x + cc[..., 2] * y + cc[..., 3] * zz + cc[..., 4] * x * x
             + cc[..., 5] * y * y + cc[..., 6] * zz * zz + cc[..., 7] * x * y + cc[..., 8] * y * zz
             + cc[..., 9] * x * zz)
        out[z0:z1] = v.to(tdt)
    n = out.numel()
    nspk = int(round(n * spike_frac))
    if nspk:
        g = torch.Generator(device=device)
        g.manual_seed(int(seed))
        idx = torch.randint(0, n, (nspk,), device=device, generator=g)
        sign = torch.where(torch.rand(nspk, device=device, generator=g) < 0.5, -1.0, 1.0)
        out.view(-1)[idx] = (sign * spike_amp).to(tdt)
    return out
