"""Seeded synthetic fields with the shapes and value distributions of the benchmark workloads.

No public dataset is available offline; these generators stand in for the SDRBench fields the
reference's integration tests name (Miranda, CESM, Hurricane).

* ``sinusoid_field``  — sum of 16 seeded 3-D sinusoids (integer wavenumbers uniform in 1..6 per
  axis, uniform phases, amplitude 1/|k|), normalised to [-1, 1], plus N(0, sigma^2) noise.
* ``spectral_field``  — Gaussian random field with isotropic power spectrum P(k) ~ k^-11/3,
  synthesised by an inverse real FFT of seeded complex white noise shaped by sqrt(P), then
  normalised to zero mean and unit variance.
* ``outlier_field``   — spectral field + linear ramp along the slowest axis + +/-100 spikes.
* ``latlon_field``    — 2-D sinusoids weighted by cos(latitude) plus noise.
"""
from __future__ import annotations

import numpy as np


def sinusoid_field(shape=(100, 200, 300), seed=0, n_waves=16, noise=1e-4, dtype=np.float32):
    rng = np.random.default_rng(seed)
    axes = [np.arange(s, dtype=np.float64) / s for s in shape]
    out = np.zeros(shape, np.float64)
    for _ in range(n_waves):
        k = rng.integers(1, 7, size=len(shape))
        phase = rng.uniform(0, 2 * np.pi)
        amp = 1.0 / np.linalg.norm(k)
        arg = np.zeros(shape, np.float64)
        for d, ax in enumerate(axes):
            sh = [1] * len(shape)
            sh[d] = -1
            arg = arg + 2 * np.pi * k[d] * ax.reshape(sh)
        out += amp * np.sin(arg + phase)
    lo, hi = out.min(), out.max()
    out = 2 * (out - lo) / (hi - lo) - 1
    out += rng.normal(0.0, noise, size=shape)
    return out.astype(dtype)


def _spectral_numpy(shape, seed):
    rng = np.random.default_rng(seed)
    rshape = list(shape[:-1]) + [shape[-1] // 2 + 1]
    noise = (rng.standard_normal(rshape, dtype=np.float32)
             + 1j * rng.standard_normal(rshape, dtype=np.float32)).astype(np.complex64)
    k2 = np.zeros(rshape, np.float32)
    for d, s in enumerate(shape):
        f = np.fft.rfftfreq(s) if d == len(shape) - 1 else np.fft.fftfreq(s)
        sh = [1] * len(shape)
        sh[d] = -1
        k2 = k2 + (f.astype(np.float32) * s).reshape(sh) ** 2
    k = np.sqrt(k2)
    k.flat[0] = 1.0
    amp = k ** (-11.0 / 6.0)      # sqrt(P), P ~ k^-11/3
    amp.flat[0] = 0.0
    noise *= amp
    try:
        import scipy.fft as sfft
        field = sfft.irfftn(noise, s=shape, workers=-1)
    except Exception:  # pragma: no cover
        field = np.fft.irfftn(noise, s=shape)
    return field


def spectral_field(shape=(512, 512, 512), seed=1, dtype=np.float32):
    field = np.asarray(_spectral_numpy(shape, seed), dtype=np.float64 if dtype == np.float64 else np.float32)
    field = field - field.mean(dtype=np.float64)
    field = field / field.std(dtype=np.float64)
    return field.astype(dtype)


def outlier_field(shape=(384, 384, 384), seed=2, ramp=10.0, spike_frac=0.005, spike=100.0, dtype=np.float64):
    x = spectral_field(shape, seed, np.float64)
    x += ramp * np.linspace(0.0, 1.0, shape[0]).reshape([-1] + [1] * (len(shape) - 1))
    rng = np.random.default_rng(seed + 1000)
    n = int(spike_frac * x.size)
    pos = rng.choice(x.size, size=n, replace=False)
    x.reshape(-1)[pos] = np.where(rng.random(n) < 0.5, -spike, spike)
    return x.astype(dtype)


def latlon_field(shape=(1800, 3600), seed=3, n_waves=16, noise=1e-3, dtype=np.float32):
    rng = np.random.default_rng(seed)
    lat = np.linspace(-np.pi / 2, np.pi / 2, shape[0]).reshape(-1, 1)
    lon = np.linspace(0, 2 * np.pi, shape[1], endpoint=False).reshape(1, -1)
    out = np.zeros(shape, np.float64)
    for _ in range(n_waves):
        k = rng.integers(1, 7, size=2)
        ph = rng.uniform(0, 2 * np.pi)
        out += np.sin(k[0] * 2 * lat + k[1] * lon + ph) / np.hypot(*k)
    out *= np.cos(lat)
    out += rng.normal(0.0, noise, size=shape)
    return out.astype(dtype)


def spectral_field_torch(shape=(512, 512, 512), seed=1, device="cuda", dtype=None):
    """The spectral (k^-11/3) Gaussian random field generated on a CUDA device with torch.

    Same construction as spectral_field (complex white noise shaped by k^-11/6, inverse real FFT,
    zero mean / unit variance), with torch's generator, so it is fast at 512^3.
    """
    import torch
    dtype = dtype or torch.float32
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    rshape = list(shape[:-1]) + [shape[-1] // 2 + 1]
    re = torch.randn(rshape, generator=g, device=device, dtype=torch.float32)
    im = torch.randn(rshape, generator=g, device=device, dtype=torch.float32)
    k2 = torch.zeros(rshape, device=device, dtype=torch.float32)
    for d, s in enumerate(shape):
        f = torch.fft.rfftfreq(s, device=device) if d == len(shape) - 1 else torch.fft.fftfreq(s, device=device)
        sh = [1] * len(shape)
        sh[d] = -1
        k2 = k2 + (f.float() * s).reshape(sh) ** 2
    k = torch.sqrt(k2)
    k.view(-1)[0] = 1.0
    amp = k ** (-11.0 / 6.0)
    amp.view(-1)[0] = 0.0
    spec = torch.complex(re * amp, im * amp)
    del re, im, k2, k, amp
    x = torch.fft.irfftn(spec, s=shape)
    del spec
    x = x.double() if dtype == torch.float64 else x
    x = (x - x.mean(dtype=torch.float64)) / x.std()
    return x.to(dtype).contiguous()


def batch_workload(n=2000, seed=4, device="cuda"):
    """The batched mixed-size workload: n fields with per-field seeds from the spectral
    generator.  60 % are 3-D cubes with side log-uniform in [16, 192], 30 % 2-D arrays with each
    side log-uniform in [64, 2048], 10 % 1-D series of length log-uniform in [4 Ki, 4 Mi]; 80 %
    float32 and 20 % float64; each with its own relative error bound, log-uniform in
    [1e-5, 1e-2].  Returns a list of (device tensor, relative error bound)."""
    import torch
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        u = rng.random()
        if u < 0.6:
            s = int(round(np.exp(rng.uniform(np.log(16), np.log(192)))))
            shape = (s, s, s)
        elif u < 0.9:
            shape = tuple(int(round(np.exp(rng.uniform(np.log(64), np.log(2048))))) for _ in range(2))
        else:
            shape = (int(round(np.exp(rng.uniform(np.log(4096), np.log(4 << 20))))),)
        dt = torch.float64 if rng.random() < 0.2 else torch.float32
        rel = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-2))))
        x = spectral_field_torch(shape, seed=seed * 100003 + i, device=device, dtype=dt)
        out.append((x, rel))
    return out
