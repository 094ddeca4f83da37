"""Synthetic XYZV fields of the benchmark shapes (the reference's datasets are
not available; these seeded fields stand in for them).

Component order. The reference's system functor returns the interpolated
sample with reversed components, dxdt = (v[2], v[1], v[0])
(particle_advector.cpp:369, "data-specific"). So that a flow u = (u_x, u_y,
u_z) moves particles along u, every generator here stores node values as
(u_z, u_y, u_x).

Noise is drawn with numpy's PCG64 from the given seed (identical on every
machine); smoothing and curls run in torch (CPU here, CUDA when a device is
given) in float64.
"""
from __future__ import annotations

import math

import numpy as np

from .advector import RegularGrid, UnsteadyGrid

ABC_A = math.sqrt(3.0)
ABC_B = math.sqrt(2.0)
ABC_C = 1.0


def _store_reversed(ux, uy, uz) -> np.ndarray:
    return np.ascontiguousarray(np.stack([uz, uy, ux], axis=-1).astype(np.float32))


def abc_velocity(x, y, z, A=ABC_A, B=ABC_B, C=ABC_C):
    """ABC flow u = (A sin z + C cos y, B sin x + A cos z, C sin y + B cos x)."""
    return (A * np.sin(z) + C * np.cos(y), B * np.sin(x) + A * np.cos(z),
            C * np.sin(y) + B * np.cos(x))


def abc(n: int, A=ABC_A, B=ABC_B, C=ABC_C, lo=0.0, hi=2.0 * math.pi) -> RegularGrid:
    """ABC flow sampled on an n^3 grid over [lo, hi]^3, spacing (hi - lo)/(n - 1)."""
    h = np.float32((hi - lo) / (n - 1))
    coords = np.float64(lo) + np.arange(n, dtype=np.float64) * np.float64(h)
    x, y, z = np.meshgrid(coords, coords, coords, indexing="ij")
    ux, uy, uz = abc_velocity(x, y, z, A, B, C)
    return RegularGrid.from_data(_store_reversed(ux, uy, uz), (h, h, h), (lo, lo, lo))


def _torch_device(device):
    import torch
    return torch.device(device) if device is not None else torch.device("cpu")


def smoothed_noise(n: int, sigma: float, seed: int, components: int = 3, device=None):
    """i.i.d. N(0, 1) noise (PCG64, `seed`) Gaussian-smoothed with standard
    deviation `sigma` cells under periodic boundaries. Returns a float64 torch
    tensor [components, n, n, n]."""
    import torch
    dev = _torch_device(device)
    rng = np.random.default_rng(seed)
    out = torch.empty((components, n, n, n), dtype=torch.float64, device=dev)
    f = torch.fft.fftfreq(n, d=1.0, device=dev, dtype=torch.float64)
    fr = torch.fft.rfftfreq(n, d=1.0, device=dev, dtype=torch.float64)
    g1 = torch.exp(-0.5 * (2.0 * math.pi * sigma * f) ** 2)
    g2 = torch.exp(-0.5 * (2.0 * math.pi * sigma * fr) ** 2)
    kernel = g1[:, None, None] * g1[None, :, None] * g2[None, None, :]
    for c in range(components):
        noise = torch.from_numpy(rng.standard_normal((n, n, n), dtype=np.float32)).to(dev)
        spec = torch.fft.rfftn(noise.to(torch.float64))
        out[c] = torch.fft.irfftn(spec * kernel, s=(n, n, n))
        del noise, spec
    return out


def _curl(psi, h: float):
    """Central-difference curl of a periodic vector potential [3, n, n, n]."""
    import torch

    def d(a, axis):
        return (torch.roll(a, -1, dims=axis) - torch.roll(a, 1, dims=axis)) / (2.0 * h)

    ux = d(psi[2], 1) - d(psi[1], 2)
    uy = d(psi[0], 2) - d(psi[2], 0)
    uz = d(psi[1], 0) - d(psi[0], 1)
    return ux, uy, uz


def curl_noise(n: int, sigma: float, seed: int, spacing: float = 1.0, device=None) -> RegularGrid:
    """Divergence-free random field: the curl of a vector potential whose
    components are smoothed N(0, 1) noise, normalized to unit RMS speed."""
    import torch
    psi = smoothed_noise(n, sigma, seed, 3, device)
    ux, uy, uz = _curl(psi, spacing)
    del psi
    rms = torch.sqrt(torch.mean(ux * ux + uy * uy + uz * uz))
    data = torch.stack([uz / rms, uy / rms, ux / rms], dim=-1).to(torch.float32)
    data = data.cpu().numpy()
    return RegularGrid.from_data(data, (spacing,) * 3, (0.0, 0.0, 0.0))


def abc_perturbed(n: int, epsilon: float = 0.05, sigma: float = 3.0, seed: int = 2,
                  device=None) -> RegularGrid:
    """ABC flow on [0, 2 pi]^3 plus a smoothed Gaussian perturbation whose RMS
    speed is `epsilon` times the ABC field's RMS speed."""
    import torch
    base = abc(n)
    h = float(base.spacing[0])
    coords = np.arange(n, dtype=np.float64) * h
    x, y, z = np.meshgrid(coords, coords, coords, indexing="ij")
    ux, uy, uz = abc_velocity(x, y, z)
    rms_abc = math.sqrt(float(np.mean(ux * ux + uy * uy + uz * uz)))
    noise = smoothed_noise(n, sigma, seed, 3, device)
    rms_noise = float(torch.sqrt(torch.mean(torch.sum(noise * noise, dim=0))))
    scale = epsilon * rms_abc / rms_noise
    noise = (noise * scale).cpu().numpy()
    data = _store_reversed(ux + noise[0], uy + noise[1], uz + noise[2])
    return RegularGrid.from_data(data, base.spacing, base.offset)


def linear(n: int, gradient: np.ndarray, constant, spacing=(1.0, 1.0, 1.0),
           offset=(0.0, 0.0, 0.0)) -> RegularGrid:
    """Field whose stored node value is constant + gradient @ (x, y, z); the
    trilinear interpolant of such a field is exact."""
    spacing = np.asarray(spacing, np.float32)
    offset = np.asarray(offset, np.float32)
    idx = np.stack(np.meshgrid(*[np.arange(n, dtype=np.float64)] * 3, indexing="ij"), axis=-1)
    xyz = offset.astype(np.float64) + idx * spacing.astype(np.float64)
    data = np.asarray(constant, np.float64) + xyz @ np.asarray(gradient, np.float64).T
    return RegularGrid.from_data(data.astype(np.float32), spacing, offset)


def double_gyre_velocity(x, y, z, t, A=0.1, epsilon=0.25, omega=2.0 * math.pi / 10.0):
    """Time-dependent double gyre on [0, 2] x [0, 1] (Shadden et al. 2005),
    with an added vertical component w = 0.1 sin(pi z):
    f(x, t) = a x^2 + b x, a = eps sin(wt), b = 1 - 2 eps sin(wt);
    u = -pi A sin(pi f) cos(pi y), v = pi A cos(pi f) sin(pi y) df/dx."""
    a = epsilon * np.sin(omega * t)
    b = 1.0 - 2.0 * epsilon * np.sin(omega * t)
    f = a * x * x + b * x
    dfdx = 2.0 * a * x + b
    u = -math.pi * A * np.sin(math.pi * f) * np.cos(math.pi * y)
    v = math.pi * A * np.cos(math.pi * f) * np.sin(math.pi * y) * dfdx
    w = 0.1 * np.sin(math.pi * z) + 0.0 * t
    return u, v, w


def double_gyre(shape=(128, 64, 64), slices: int = 32, period: float = 10.0, A=0.1,
                epsilon=0.25) -> UnsteadyGrid:
    """The double gyre sampled on [0, 2] x [0, 1] x [0, 1] with `slices` time
    slices spanning one period [0, period] (slice spacing period / (slices - 1))."""
    n = shape
    h = np.array([2.0 / (n[0] - 1), 1.0 / (n[1] - 1), 1.0 / (n[2] - 1)], np.float32)
    x = np.arange(n[0], dtype=np.float64)[:, None, None] * np.float64(h[0])
    y = np.arange(n[1], dtype=np.float64)[None, :, None] * np.float64(h[1])
    z = np.arange(n[2], dtype=np.float64)[None, None, :] * np.float64(h[2])
    dt = np.float32(period / (slices - 1))
    data = np.empty((slices,) + tuple(n) + (3,), np.float32)
    for s in range(slices):
        t = np.float64(np.float32(s) * dt)
        u, v, w = double_gyre_velocity(x, y, z, t, A, epsilon, 2.0 * math.pi / period)
        u, v, w = np.broadcast_arrays(u, v, w)
        data[s] = _store_reversed(u, v, w)
    return UnsteadyGrid.from_data(data, h, float(dt))
