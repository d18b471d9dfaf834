"""Seeded synthetic fields that stand in for the scientific datasets the
compressor is benchmarked on (the reference quotes public simulation fields
that are not available offline). Every generator is deterministic for a seed.

numpy generators (float64 internally, then cast) serve the small parity
cases; the ``device=`` variants build the same kind of field with torch on a
GPU, for the 100M-sample workloads where host FFTs would dominate a run.
"""
from __future__ import annotations

import math

import numpy as np


def sinusoids(shape=(64, 64, 64), seed=0, waves=8, noise=1e-3, dtype=np.float32):
    """Sum of random 3D sinusoids plus Gaussian noise; shape is (z, y, x).

    Wavenumbers uniform in [1, 6] per axis, amplitudes uniform in [0.1, 1],
    phases uniform in [0, 2*pi), noise N(0, noise**2)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")
    field = np.zeros(shape, np.float64)
    for _ in range(waves):
        kx, ky, kz = rng.uniform(1.0, 6.0, 3)
        amp = rng.uniform(0.1, 1.0)
        phase = rng.uniform(0.0, 2 * math.pi)
        field += amp * np.sin(2 * math.pi * (kx * x + ky * y + kz * z) + phase)
    field += rng.normal(0.0, noise, shape)
    return field.astype(dtype)


def _spectral_amplitude(shape, slope):
    nz, ny, nx = shape
    kz = np.fft.fftfreq(nz) * nz
    ky = np.fft.fftfreq(ny) * ny
    kx = np.fft.rfftfreq(nx) * nx
    k = np.sqrt(kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
    amp = np.zeros_like(k)
    nz_mask = k > 0
    amp[nz_mask] = k[nz_mask] ** (slope / 2.0)  # power ~ k^slope -> amplitude k^(slope/2)
    return amp


def power_law_field(shape, seed, slope=-11.0 / 3.0, dtype=np.float32):
    """Gaussian random field with power spectrum ~ |k|^slope, unit variance."""
    rng = np.random.Generator(np.random.PCG64(seed))
    white = rng.standard_normal(shape)
    spec = np.fft.rfftn(white) * _spectral_amplitude(shape, slope)
    field = np.fft.irfftn(spec, s=shape, axes=tuple(range(len(shape))))
    field -= field.mean()
    field /= field.std()
    return field.astype(dtype)


def power_law_field_device(shape, seed, slope=-11.0 / 3.0, dtype=None, device="cuda"):
    """Same construction as power_law_field with torch on a GPU (fp64 FFTs)."""
    import torch
    dtype = dtype or torch.float32
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    nz, ny, nx = shape
    white = torch.randn(shape, generator=g, device=device, dtype=torch.float64)
    spec = torch.fft.rfftn(white)
    del white
    kz = torch.fft.fftfreq(nz, device=device, dtype=torch.float64) * nz
    ky = torch.fft.fftfreq(ny, device=device, dtype=torch.float64) * ny
    kx = torch.fft.rfftfreq(nx, device=device, dtype=torch.float64) * nx
    k2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    amp = torch.where(k2 > 0, k2.clamp_min(1e-300) ** (slope / 4.0), torch.zeros_like(k2))
    spec *= amp
    del amp, k2
    field = torch.fft.irfftn(spec, s=shape)
    del spec
    field -= field.mean()
    field /= field.std()
    return field.to(dtype)


def front_field(shape=(96, 256, 384), seed=2, dtype=np.float64):
    """Smooth k^-5/3 field plus a sharp front 10*tanh((z-48)/2) along z."""
    base = power_law_field(shape, seed, slope=-5.0 / 3.0, dtype=np.float64)
    z = np.arange(shape[0], dtype=np.float64)[:, None, None]
    return (base + 10.0 * np.tanh((z - shape[0] / 2) / 2.0)).astype(dtype)


def spiky_field(shape=(64, 1024, 1024), seed=3, fraction=0.01, magnitude=50.0, dtype=np.float32):
    """k^-11/3 field with a given fraction of samples replaced by +-magnitude."""
    field = power_law_field(shape, seed, dtype=np.float64)
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    n = field.size
    idx = rng.choice(n, int(n * fraction), replace=False)
    field.reshape(-1)[idx] = np.where(rng.random(idx.size) < 0.5, -magnitude, magnitude)
    return field.astype(dtype)


def spiky_field_device(shape=(64, 1024, 1024), seed=3, fraction=0.01, magnitude=50.0, device="cuda"):
    """spiky_field built with torch on a GPU: a device k^-11/3 field (seed)
    with each sample replaced by +-magnitude with probability `fraction`
    (signs equally likely), from a torch generator seeded with `seed`.
    Returns a contiguous float32 CUDA tensor."""
    import torch
    f = power_law_field_device(shape, seed, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    spikes = torch.rand(shape, device=device, generator=gen) < fraction
    signs = torch.where(torch.rand(shape, device=device, generator=gen) < 0.5, -magnitude, magnitude)
    return torch.where(spikes, signs, f).to(torch.float32).contiguous()


def uneven_chunks(count=512, seed=4, sides=(32, 48, 64, 96, 128), dtype=np.float32):
    """List of k^-11/3 chunks with per-axis sides drawn from `sides` and each
    chunk rescaled to a value range drawn log-uniformly in [1e-2, 1e3]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        shape = tuple(int(s) for s in rng.choice(sides, 3))
        f = power_law_field(shape, seed * 100003 + i, dtype=np.float64)
        span = 10 ** rng.uniform(-2, 3)
        lo, hi = f.min(), f.max()
        f = (f - lo) / (hi - lo) * span
        out.append(f.astype(dtype))
    return out


def uneven_chunks_device(count=512, seed=4, sides=(32, 48, 64, 96, 128), device="cuda"):
    """uneven_chunks built with torch on a GPU: the same shape and value-range
    draws (numpy PCG64 stream of `seed`), device-generated k^-11/3 fields.
    Returns float32 CUDA tensors."""
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        shape = tuple(int(s) for s in rng.choice(sides, 3))
        f = power_law_field_device(shape, seed * 100003 + i, dtype=torch.float64, device=device)
        span = 10 ** rng.uniform(-2, 3)
        lo, hi = f.min(), f.max()
        out.append(((f - lo) / (hi - lo) * span).to(torch.float32).contiguous())
    return out


def rel_to_abs(field, rel: float) -> float:
    """REL bound -> absolute bound: rel * (max - min) evaluated in double."""
    lo = float(field.min())
    hi = float(field.max())
    return rel * (hi - lo)
