"""Initial conditions injected on the host (FP64 numpy), shape (nz, ny, nx).

The reference builds its ICs with operators (source/operators/InitialConditions.cpp:20-230,
source/spectralOperators/SpectralIcGenerator.cpp:21-135); the workloads here
are injected directly:
  * Taylor-Green: u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 at cell centres;
  * decaying turbulence: seeded random Fourier amplitudes with
    E(k) ~ k^4 exp(-2 (k/k0)^2) (the shape of SpectralIcGenerator.cpp:75-80 with
    k0 = 4), uniform random phases, projected onto the discretely solenoidal
    fields (central divergence zero, the wide-stencil projection the solver
    uses) and scaled to u_rms = 1;
  * a seeded Gaussian solenoidal perturbation band-limited to |k| <= kmax.
"""
from __future__ import annotations

import numpy as np


def cell_centres(cells, h):
    nx, ny, nz = cells
    x = (np.arange(nx) + 0.5) * h
    y = (np.arange(ny) + 0.5) * h
    z = (np.arange(nz) + 0.5) * h
    return np.meshgrid(z, y, x, indexing="ij")  # Z, Y, X each (nz, ny, nx)


def taylor_green(cells, h):
    Z, Y, X = cell_centres(cells, h)
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    return u, v, w


def _wavenumbers(shape):
    nz, ny, nx = shape
    kz = np.fft.fftfreq(nz, 1.0 / nz)[:, None, None]
    ky = np.fft.fftfreq(ny, 1.0 / ny)[None, :, None]
    kx = np.fft.rfftfreq(nx, 1.0 / nx)[None, None, :]
    return kz, ky, kx


def project_discrete_solenoidal(u, v, w):
    """Removes the central-difference gradient part: after this, the central
    divergence (u(x+1) - u(x-1) + ...) vanishes to rounding."""
    shape = u.shape
    nz, ny, nx = shape
    kz, ky, kx = _wavenumbers(shape)
    sx = np.sin(2 * np.pi * kx / nx) + 0 * kz + 0 * ky
    sy = np.sin(2 * np.pi * ky / ny) + 0 * kz + 0 * kx
    sz = np.sin(2 * np.pi * kz / nz) + 0 * ky + 0 * kx
    U, V, W = (np.fft.rfftn(a, axes=(0, 1, 2)) for a in (u, v, w))
    s2 = sx * sx + sy * sy + sz * sz
    with np.errstate(divide="ignore", invalid="ignore"):
        dot = (sx * U + sy * V + sz * W) / s2
    dot[s2 == 0] = 0
    U, V, W = U - sx * dot, V - sy * dot, W - sz * dot
    return tuple(np.fft.irfftn(a, s=shape, axes=(0, 1, 2)) for a in (U, V, W))


def random_solenoidal(cells, seed, spectrum, kmax=None, rms=None, amplitude=None):
    """Random field with E(k) ~ spectrum(k), random phases, discretely solenoidal."""
    nx, ny, nz = cells
    shape = (nz, ny, nx)
    rng = np.random.Generator(np.random.PCG64(seed))
    kz, ky, kx = _wavenumbers(shape)
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.sqrt(spectrum(k) / (4 * np.pi * np.maximum(k, 1e-30) ** 2))
    amp[k == 0] = 0
    if kmax is not None:
        amp[k > kmax] = 0
    comps = []
    for _ in range(3):
        phase = rng.uniform(0, 2 * np.pi, size=amp.shape)
        mag = rng.standard_normal(size=amp.shape)
        comps.append(np.fft.irfftn(amp * mag * np.exp(1j * phase), s=shape, axes=(0, 1, 2)))
    u, v, w = project_discrete_solenoidal(*comps)
    if rms is not None:
        cur = np.sqrt(np.mean(u * u + v * v + w * w) / 3.0)
        u, v, w = (a * (rms / cur) for a in (u, v, w))
    if amplitude is not None:
        cur = np.sqrt(np.mean(u * u + v * v + w * w) / 3.0)
        u, v, w = (a * (amplitude / cur) for a in (u, v, w))
    return u, v, w


def decaying_turbulence(cells, seed=1234, k0=4.0):
    return random_solenoidal(cells, seed, lambda k: k ** 4 * np.exp(-2.0 * (k / k0) ** 2), rms=1.0)


def perturbed_taylor_green(cells, h, seed, amplitude=0.05, kmax=8):
    u, v, w = taylor_green(cells, h)
    du, dv, dw = random_solenoidal(cells, seed, lambda k: np.ones_like(k), kmax=kmax, amplitude=amplitude)
    return u + du, v + dv, w + dw
