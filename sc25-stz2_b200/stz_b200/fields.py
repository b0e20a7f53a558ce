"""Seeded synthetic 3-D fields with the shapes and value distributions of the
benchmark workloads (the reference's SDRBench datasets are not available):

* grf(shape, alpha)   Gaussian random field: white noise filtered in Fourier
                      space to power spectrum P(k) ~ k^-alpha, zero mean,
                      unit variance.
* lognormal(shape)    exp(1.5 g), g a unit GRF with P(k) ~ k^-3.
* fronts(shape)       GRF with P(k) ~ k^-5/3 plus 20 planar tanh shear fronts
                      (random normals, width U[2,8] cells, amplitude 3 sigma).

Each has a numpy implementation (small sizes, tests) and a torch one
(`device=` a CUDA device, for the 512^3 - 1024^3 benchmark fields).
"""
from __future__ import annotations

import numpy as np


def _kmag_np(shape):
    kz = np.fft.fftfreq(shape[0])[:, None, None]
    ky = np.fft.fftfreq(shape[1])[None, :, None]
    kx = np.fft.rfftfreq(shape[2])[None, None, :]
    return np.sqrt(kz * kz + ky * ky + kx * kx)


def grf(shape, alpha: float, seed: int, dtype=np.float32, device=None):
    if device is not None:
        return _grf_torch(shape, alpha, seed, dtype, device)
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    f = np.fft.rfftn(w)
    k = _kmag_np(shape)
    k[0, 0, 0] = 1.0
    f *= k ** (-alpha / 2.0)
    f[0, 0, 0] = 0.0
    g = np.fft.irfftn(f, s=shape, axes=(0, 1, 2))
    g -= g.mean()
    g /= g.std()
    return g.astype(dtype)


def _grf_torch(shape, alpha, seed, dtype, device):
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    w = torch.randn(shape, generator=gen, device=device, dtype=torch.float32)
    f = torch.fft.rfftn(w)
    del w
    kz = torch.fft.fftfreq(shape[0], device=device)[:, None, None]
    ky = torch.fft.fftfreq(shape[1], device=device)[None, :, None]
    kx = torch.fft.rfftfreq(shape[2], device=device)[None, None, :]
    k = torch.sqrt(kz * kz + ky * ky + kx * kx)
    k[0, 0, 0] = 1.0
    f *= k.pow(-alpha / 2.0)
    f[0, 0, 0] = 0.0
    del k
    g = torch.fft.irfftn(f, s=shape)
    del f
    g -= g.mean()
    g /= g.std()
    tdt = {np.float32: torch.float32, np.float64: torch.float64}[np.dtype(dtype).type]
    return g.to(tdt).contiguous()


def lognormal(shape, seed: int, dtype=np.float32, device=None):
    g = grf(shape, 3.0, seed, np.float64 if device is None else np.float32, device)
    if device is not None:
        import torch

        out = torch.exp(1.5 * g)
        return out.to({np.float32: torch.float32, np.float64: torch.float64}[np.dtype(dtype).type]).contiguous()
    return np.exp(1.5 * g).astype(dtype)


def fronts(shape, seed: int, dtype=np.float64, n_fronts: int = 20, device=None):
    g = grf(shape, 5.0 / 3.0, seed, np.float64, None if device is None else device)
    rng = np.random.default_rng(seed + 7919)
    nz, ny, nx = shape
    if device is not None:
        import torch

        z = torch.arange(nz, device=device, dtype=torch.float64)[:, None, None]
        y = torch.arange(ny, device=device, dtype=torch.float64)[None, :, None]
        x = torch.arange(nx, device=device, dtype=torch.float64)[None, None, :]
        out = g.to(torch.float64)
        for _ in range(n_fronts):
            nv = rng.standard_normal(3)
            nv /= np.linalg.norm(nv)
            c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
            w = rng.uniform(2, 8)
            s = (x - c[0]) * nv[0] + (y - c[1]) * nv[1] + (z - c[2]) * nv[2]
            out += 3.0 * torch.tanh(s / w)
        return out.to({np.float32: torch.float32, np.float64: torch.float64}[np.dtype(dtype).type]).contiguous()
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = g.astype(np.float64)
    for _ in range(n_fronts):
        nv = rng.standard_normal(3)
        nv /= np.linalg.norm(nv)
        c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
        w = rng.uniform(2, 8)
        s = (x - c[0]) * nv[0] + (y - c[1]) * nv[1] + (z - c[2]) * nv[2]
        out += 3.0 * np.tanh(s / w)
    return out.astype(dtype)
