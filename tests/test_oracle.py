"""CPU tests of the oracle (the FP64 restatement used as the parity checker).

Pins: the periodic lab semantics against the restated
tests/cubismup3d/TestBoundaries.cpp, the FFT Poisson solve against numpy's
pocketfft (FFTW 3.3.7's DFT definition) and the committed golden vectors,
plus analytic known answers.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def element_value(x, y, z):
    # tests/cubismup3d/TestBoundaries.cpp:13-16
    return x + 1000 * y + 1000000 * z


@pytest.mark.parametrize("g,shift", [(1, (-1, 0, 0)), (1, (+1, 0, 0)), (2, (-1, +1, +2))])
def test_periodic_lab_test_boundaries(oracle, g, shift):
    # tests/cubismup3d/TestBoundaries.cpp:55-75: 128x32x32 periodic grid.
    nx, ny, nz = 128, 32, 32
    Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    f = element_value(X, Y, Z).astype(np.float64)
    dx, dy, dz = shift
    out = oracle.lab_shift(f, g, dx, dy, dz)
    expected = element_value((X - dx) % nx, (Y - dy) % ny, (Z - dz) % nz)
    assert np.array_equal(out, expected)


def numpy_poisson(rhs, h):
    """Independent restatement of PoissonSolverPeriodic::solve with numpy's
    pocketfft in FFTW's layout (x slowest, z r2c last)."""
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


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 16, 64), (64, 32, 16)])
def test_poisson_matches_pocketfft(oracle, shape):
    rng = np.random.default_rng(7)
    rhs = rng.standard_normal(shape)
    h = 0.37
    p = oracle.poisson_solve(rhs, h)
    assert rel_l2(p, numpy_poisson(rhs, h)) < 1e-13


def test_poisson_golden_vectors(oracle):
    d = np.load(os.path.join(GOLDEN, "poisson_golden.npz"))
    for key in ("a", "b"):
        rhs, h, p = d[f"{key}_rhs"], float(d[f"{key}_h"]), d[f"{key}_p"]
        assert rel_l2(oracle.poisson_solve(rhs, h), p) < 1e-13


def wide_laplacian(p, h):
    out = np.zeros_like(p)
    for ax in range(3):
        out += (np.roll(p, -2, ax) - 2 * p + np.roll(p, 2, ax)) / (4 * h * h)
    return out


def test_poisson_single_mode_known_answer(oracle):
    # rhs = h^3 cos(2 pi (a x / nx + b y / ny + c z / nz)): p = rhs / (h^3 lambda),
    # lambda = sum_d (2 cos(4 pi k_d / N_d) - 2) / (4 h^2).
    nz, ny, nx = 16, 32, 64
    h = 0.1
    Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    a, b, c = 3, 5, 2
    phase = 2 * np.pi * (a * X / nx + b * Y / ny + c * Z / nz)
    rhs = h ** 3 * np.cos(phase)
    lam = sum((2 * np.cos(4 * np.pi * k / n) - 2) / (4 * h * h) for k, n in ((a, nx), (b, ny), (c, nz)))
    p = oracle.poisson_solve(rhs, h)
    assert rel_l2(p, np.cos(phase) / lam) < 1e-13
    assert rel_l2(wide_laplacian(p, h) * h ** 3, rhs) < 1e-12


def test_projection_makes_divergence_free(oracle):
    from cubismup_3d_b200 import initial_conditions as ic
    n = 32
    h = 2 * np.pi / n
    sim = oracle.OracleSim(n, n, n, 2 * np.pi, nu=0.01, CFL=0.5, rampup=0, DLM=0.0, lambda_=1.0)
    u, v, w = ic.random_solenoidal((n, n, n), 3, lambda k: np.exp(-k), rms=1.0)
    u = u + 0.3 * np.sin(np.arange(n) * h)[None, None, :]  # add a divergent part
    sim.set_velocity(u, v, w)
    d0 = sim.diagnostics()["div_l2"]
    dt = 0.01
    sim.operator("AdvectionDiffusion", dt)
    sim.operator("PressureRHS", dt)
    sim.operator("PressureProjection", dt)
    d1 = sim.diagnostics()
    assert d0 > 1e-2
    assert d1["div_l2"] < 1e-12 * max(1.0, d0)


def test_taylor_green_viscous_decay(oracle):
    # small dt, pure TG: KE decays like exp(-2 * 3 nu t) to leading order (the
    # central-difference modified wavenumber makes it a little slower).
    from cubismup_3d_b200 import initial_conditions as ic
    n = 32
    h = 2 * np.pi / n
    nu = 0.05
    sim = oracle.OracleSim(n, n, n, 2 * np.pi, nu=nu, CFL=0.1, rampup=0, DLM=0.0, lambda_=1.0)
    sim.set_velocity(*ic.taylor_green((n, n, n), h))
    ke0 = sim.diagnostics()["ke"]
    dts = sim.run(20)
    ke1 = sim.diagnostics()["ke"]
    t = float(np.sum(dts))
    ratio = ke1 / ke0
    assert np.exp(-6 * nu * t) < ratio < 1.0
    assert abs(ratio - np.exp(-6 * nu * t)) < 0.02


def test_calc_max_timestep_rampup(oracle):
    n = 16
    sim = oracle.OracleSim(n, n, n, 1.0, nu=0.01, CFL=0.5, rampup=10, DLM=1.0, lambda_=1.0)
    u = np.full((n, n, n), 0.5)
    sim.set_velocity(u, 0 * u, 0 * u)
    dt = sim.calc_max_timestep()
    h = 1.0 / n
    base = min(h * h / 0.01, h / (0.5 + 1e-8))
    x = 1.0 / 10
    ramp = np.exp(np.log(1e-3) * (1 - x) + np.log(0.5) * x)
    assert dt == pytest.approx(ramp * base, rel=1e-15)
    assert sim.stats()["lambda"] == pytest.approx(1.0 / dt, rel=1e-15)


def test_sphere_chi_and_penalization(oracle):
    # sphere at rest in a fixed frame: chi in [0,1], CoM at the centre, and the
    # implicit penalization pulls the velocity inside the body to U_s.
    n = 32
    sphere = {"radius": 0.2, "position": (0.5, 0.5, 0.5), "velocity": (1.0, 0, 0), "forced": (1, 1, 1),
              "fix_frame": (1, 1, 1)}
    sim = oracle.OracleSim(n, n, n, 1.0, nu=0.01, CFL=0.1, rampup=0, DLM=0.0, lambda_=1e6,
                           implicit_penalization=True, sphere=sphere)
    chi = sim.get("chi")
    st = sim.stats()
    assert chi.min() >= 0 and chi.max() <= 1 + 1e-12
    assert np.allclose(st["com"], 0.5, atol=1e-12)
    assert np.allclose(st["uinf"], (-1, 0, 0))
    vol = chi.sum() / n ** 3
    assert abs(vol - 4 / 3 * np.pi * 0.2 ** 3) / (4 / 3 * np.pi * 0.2 ** 3) < 0.02
    dts = sim.run(2)
    u = sim.get("u")
    inside = chi >= 1.0
    assert np.allclose(u[inside], 1.0, atol=1e-4)
    assert st["force"].shape == (3,)
    assert np.all(np.isfinite(sim.stats()["force"]))
    assert dts[0] > 0


@pytest.mark.parametrize("scheme", ["ref", "upwind3_rk2"])
def test_tangent_linear_matches_central_differences(oracle, scheme):
    # the FP64 tangent-linear model (checker of the GPU adjoint) against central
    # differences of the oracle forward with the same fixed dt sequence. The
    # upwind stencil switches with the sign of the advecting velocity, so its FD
    # error is O(eps) from cells that flip direction: eps is taken small there.
    from cubismup_3d_b200 import initial_conditions as ic
    n, L, nsteps = 32, 2 * np.pi, (4 if scheme == "ref" else 2)
    kw = dict(nu=5e-3, CFL=0.3, rampup=0, DLM=0.0, lambda_=1.0, scheme=scheme)
    u0 = ic.perturbed_taylor_green((n, n, n), L / n, seed=1)
    base = oracle.OracleSim(n, n, n, L, **kw)
    base.set_velocity(*u0)
    dts = base.run(nsteps)
    rng = np.random.default_rng(3)
    d = [rng.standard_normal((n, n, n)) for _ in range(3)]
    tl = oracle.OracleSim(n, n, n, L, **kw)
    tl.set_velocity(*u0)
    tang = tl.tangent_run(dts, *d)
    eps = 1e-5 if scheme == "ref" else 1e-7
    out = []
    for sgn in (+1, -1):
        s = oracle.OracleSim(n, n, n, L, **kw)
        s.set_velocity(*[a + sgn * eps * b for a, b in zip(u0, d)])
        s.run(nsteps, fixed_dts=dts)
        out.append(s.velocity())
    fd = [(a - b) / (2 * eps) for a, b in zip(*out)]
    for a, b in zip(tang, fd):
        assert rel_l2(a, b) < 1e-6


def test_moving_sphere_advances_with_its_velocity(oracle):
    # bFixFrameOfRef off: uinf = 0 (updateUinf) and every step moves the sphere
    # by dt U (Obstacle::update) before chi is rebuilt; the grid CoM follows
    n = 32
    sphere = {"radius": 0.15, "position": (0.4, 0.5, 0.5), "velocity": (1.0, 0.5, 0.0), "forced": (1, 1, 1),
              "fix_frame": (0, 0, 0)}
    sim = oracle.OracleSim(n, n, n, 1.0, nu=0.01, CFL=0.1, rampup=0, DLM=0.0, lambda_=1e6,
                           implicit_penalization=True, sphere=sphere)
    com0 = sim.stats()["com"].copy()
    assert np.allclose(sim.stats()["uinf"], 0.0)
    dts = sim.run(4)
    shift = sim.stats()["com"] - com0
    travelled = np.sum(dts) * np.array([1.0, 0.5, 0.0])
    # the CoM of the discrete chi tracks the position to a fraction of a cell
    assert np.allclose(shift, travelled, atol=0.1 / n)


def test_dissipation_sums_vs_numpy(oracle):
    # ComputeDissipation's linear and quadratic sums restated in numpy on the
    # oracle's own fields (periodic central differences)
    n, L = 32, 2 * np.pi
    sim = oracle.OracleSim(n, n, n, L, nu=0.01, CFL=0.3, rampup=0, DLM=0.0, lambda_=1.0)
    rng = np.random.default_rng(3)
    u, v, w = (rng.standard_normal((n, n, n)) for _ in range(3))
    sim.set_velocity(u, v, w)
    sim.run(2)
    d = sim.dissipation()
    u, v, w, p = (sim.get(k) for k in ("u", "v", "w", "p"))
    h = L / n
    h3 = h ** 3

    def dd(f, ax):
        return (np.roll(f, -1, ax) - np.roll(f, 1, ax)) / (2 * h)

    wx, wy, wz = dd(w, 1) - dd(v, 0), dd(u, 0) - dd(w, 2), dd(v, 2) - dd(u, 1)
    assert d[18] == pytest.approx(h3 * 0.5 * np.sum(u * u + v * v + w * w), rel=1e-12)  # kineticEn
    assert np.allclose(d[6:9], [h3 * u.sum(), h3 * v.sum(), h3 * w.sum()], rtol=1e-10, atol=1e-12)  # linMom
    assert np.allclose(d[0:3], [h3 * wx.sum(), h3 * wy.sum(), h3 * wz.sum()], atol=1e-10)  # circulation ~ 0
    assert d[17] == pytest.approx(h3 * np.sum(wx * u + wy * v + wz * w), rel=1e-9, abs=1e-9)  # helicity
    assert d[19] == pytest.approx(np.sum(np.sqrt(wx * wx + wy * wy + wz * wz)), rel=1e-12)  # enstrophy
    pres = -h3 * np.sum(dd(p, 2) * u + dd(p, 1) * v + dd(p, 0) * w)
    assert d[15] == pytest.approx(pres, rel=1e-9, abs=1e-12)  # presPow


def test_spectral_restatement_parseval(oracle):
    # the r2c restatement of the HIT statistics against physical-space
    # identities: tke = <|u|^2> / 2, eps = nu <|curl_c u|^2>; the forcing band
    # field carries exactly tke_filtered
    rng = np.random.default_rng(5)
    shape = (16, 32, 32)
    u, v, w = (rng.standard_normal(shape) for _ in range(3))
    h, nu = 0.1, 0.02
    st, E, filt = oracle.spectral(u, v, w, h, nu, band=True)
    assert st["tke"] == pytest.approx(0.5 * np.mean(u * u + v * v + w * w), rel=1e-12)

    def dd(f, ax):
        return (np.roll(f, -1, ax) - np.roll(f, 1, ax)) / (2 * h)

    wx, wy, wz = dd(w, 1) - dd(v, 0), dd(u, 0) - dd(w, 2), dd(v, 2) - dd(u, 1)
    assert st["eps"] == pytest.approx(nu * np.mean(wx * wx + wy * wy + wz * wz), rel=1e-12)
    N = u.size
    fu, fv, fw = (f / N for f in filt)
    assert st["tke_filtered"] == pytest.approx(0.5 * np.mean(fu * fu + fv * fv + fw * fw), rel=1e-10)
    assert len(E) == max(shape) // 2 - 1 and np.all(E >= 0) and E.sum() <= st["tke"]
