"""Generates tests/golden/poisson_golden.npz.

Golden vectors for PoissonSolverPeriodic::solve (source/poisson/PoissonSolverPeriodic.cpp:15-146)
computed with an independent restatement on numpy's pocketfft (FFTW's r2c/c2r
layout: x slowest, z the half-spectrum axis). The reference itself cannot be
built in this image, so these pin the oracle to the published DFT definition
rather than to reference outputs. Run: python tests/golden/make_golden.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def solve(rhs, h):
    nz, ny, nx = rhs.shape
    B = np.fft.rfftn(rhs.transpose(2, 1, 0), axes=(0, 1, 2))
    i = np.arange(nx)[:, None, None]
    l = np.arange(ny)[None, :, None]
    k = np.arange(nz // 2 + 1)[None, None, :]
    D = np.cos(4 * np.pi / nx * i) + np.cos(4 * np.pi / ny * l) + np.cos(4 * np.pi / nz * k)
    with np.errstate(divide="ignore", invalid="ignore"):
        fac = 4 / (nx * h * ny * nz) / (2 * D - 6)
        B = B * fac
    for a in (0, nx // 2):
        for c in (0, ny // 2):
            for d in (0, nz // 2):
                B[a, c, d] = 0
    return (np.fft.irfftn(B, s=(nx, ny, nz), axes=(0, 1, 2)) * (nx * ny * nz)).transpose(2, 1, 0)


def main():
    rng = np.random.Generator(np.random.PCG64(20240611))
    out = {}
    for key, shape, h in (("a", (8, 8, 16), 0.25), ("b", (4, 16, 8), 0.1)):
        rhs = rng.standard_normal(shape)
        out[f"{key}_rhs"] = rhs
        out[f"{key}_h"] = np.float64(h)
        out[f"{key}_p"] = solve(rhs, h)
    np.savez_compressed(os.path.join(HERE, "poisson_golden.npz"), **out)


if __name__ == "__main__":
    main()
