"""ORACLE — test infrastructure only.

ctypes binding of ``oracle/liboracle.so``, the CPU FP64 restatement of
CubismUP_3D's periodic fractional-step time step (see ``cup_oracle.cpp`` for
the reference file:line of every kernel and for the parity status). Only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import this
module; the product package never does.

Fields are numpy float64 arrays of shape (nz, ny, nx), x fastest, the same
global layout the CUDA library uses.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class OrcConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("maxextent", C.c_double),
        ("nu", C.c_double), ("CFL", C.c_double), ("lambda_", C.c_double), ("DLM", C.c_double),
        ("uinf", C.c_double * 3),
        ("rampup", C.c_int),
        ("implicit_penalization", C.c_int),
        ("scheme", C.c_int),
        ("has_sphere", C.c_int),
        ("sphere_radius", C.c_double),
        ("sphere_position", C.c_double * 3),
        ("sphere_velocity", C.c_double * 3),
        ("sphere_forced", C.c_int * 3),
        ("sphere_fix_frame", C.c_int * 3),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.orc_create.argtypes = [C.POINTER(OrcConfig)]
        L.orc_create.restype = C.c_void_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_h.argtypes = [C.c_void_p]
        L.orc_h.restype = C.c_double
        L.orc_set_velocity.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_get_field.argtypes = [C.c_void_p, C.c_int, dp]
        L.orc_calc_max_timestep.argtypes = [C.c_void_p]
        L.orc_calc_max_timestep.restype = C.c_double
        L.orc_max_u.argtypes = [C.c_void_p]
        L.orc_max_u.restype = C.c_double
        L.orc_operator.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
        L.orc_operator.restype = C.c_int
        L.orc_timestep.argtypes = [C.c_void_p, C.c_double]
        L.orc_run.argtypes = [C.c_void_p, C.c_int, dp, dp]
        L.orc_get_stats.argtypes = [C.c_void_p, dp]
        L.orc_poisson_solve_field.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, dp, dp]
        L.orc_poisson_solve_field.restype = C.c_int
        L.orc_lab_shift.argtypes = [dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_lab_shift.restype = C.c_int
        L.orc_diagnostics.argtypes = [C.c_void_p, dp]
        L.orc_dissipation.argtypes = [C.c_void_p, dp]
        L.orc_compute_forces.argtypes = [C.c_void_p, dp]
        L.orc_tangent_run.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, dp]
        L.orc_tangent_run.restype = C.c_int
        L.orc_num_threads.restype = C.c_int
        L.orc_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


FIELDS = {"u": 0, "v": 1, "w": 2, "p": 3, "chi": 4, "tmpU": 5, "tmpV": 6, "tmpW": 7, "rhs": 8}


class OracleSim:
    """One oracle simulation (the hot-path subset of SimulationData + pipeline)."""

    def __init__(self, nx, ny, nz, maxextent, nu, CFL=0.1, lambda_=1e6, DLM=0.0,
                 uinf=(0.0, 0.0, 0.0), rampup=0, implicit_penalization=True, scheme="ref",
                 sphere=None):
        cfg = OrcConfig()
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.maxextent = maxextent
        cfg.nu, cfg.CFL, cfg.lambda_, cfg.DLM = nu, CFL, lambda_, DLM
        cfg.uinf[:] = list(uinf)
        cfg.rampup = rampup
        cfg.implicit_penalization = int(bool(implicit_penalization))
        cfg.scheme = {"ref": 0, "upwind3_rk2": 1}[scheme]
        if sphere is not None:
            cfg.has_sphere = 1
            cfg.sphere_radius = sphere["radius"]
            cfg.sphere_position[:] = list(sphere["position"])
            cfg.sphere_velocity[:] = list(sphere.get("velocity", (0, 0, 0)))
            cfg.sphere_forced[:] = [int(x) for x in sphere.get("forced", (1, 1, 1))]
            cfg.sphere_fix_frame[:] = [int(x) for x in sphere.get("fix_frame", (0, 0, 0))]
        self.shape = (nz, ny, nx)
        self._h = lib().orc_create(C.byref(cfg))
        if not self._h:
            raise ValueError("oracle: invalid configuration")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    @property
    def h(self) -> float:
        return lib().orc_h(self._h)

    def set_velocity(self, u, v, w):
        u, v, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w))
        lib().orc_set_velocity(self._h, _p(u), _p(v), _p(w))

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        lib().orc_get_field(self._h, FIELDS[name], _p(out))
        return out

    def velocity(self):
        return self.get("u"), self.get("v"), self.get("w")

    def calc_max_timestep(self) -> float:
        return lib().orc_calc_max_timestep(self._h)

    def max_u(self) -> float:
        return lib().orc_max_u(self._h)

    def operator(self, name: str, dt: float):
        if lib().orc_operator(self._h, name.encode(), dt) != 0:
            raise ValueError(f"oracle: unknown operator {name}")

    def timestep(self, dt: float):
        lib().orc_timestep(self._h, dt)

    def run(self, nsteps: int, fixed_dts=None) -> np.ndarray:
        dts = np.zeros(nsteps, dtype=np.float64)
        fx = None
        if fixed_dts is not None:
            fx = np.ascontiguousarray(fixed_dts, dtype=np.float64)
        lib().orc_run(self._h, nsteps, _p(fx) if fx is not None else None, _p(dts))
        return dts

    def tangent_run(self, dts, du, dv, dw):
        """FP64 tangent-linear rollout with a fixed dt sequence: advances the state and
        returns the propagated tangent (du, dv, dw)."""
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        t = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in (du, dv, dw)]
        if lib().orc_tangent_run(self._h, len(dts), _p(dts), _p(t[0]), _p(t[1]), _p(t[2])) != 0:
            raise ValueError("oracle: tangent rollout does not support obstacles")
        return tuple(t)

    def stats(self) -> dict:
        out = np.zeros(34, dtype=np.float64)
        lib().orc_get_stats(self._h, _p(out))
        return {
            "force": out[0:3].copy(), "torque": out[3:6].copy(), "time": out[6], "step": int(out[7]),
            "uinf": out[8:11].copy(), "dt": out[11], "lambda": out[12], "com": out[13:16].copy(),
            "rhs_sums": out[16:19].copy(), "corr": out[19], "umax": out[20], "transVel": out[21:24].copy(),
            "angVel": out[24:27].copy(), "position": out[27:30].copy(), "quaternion": out[30:34].copy(),
        }

    def diagnostics(self) -> dict:
        out = np.zeros(3, dtype=np.float64)
        lib().orc_diagnostics(self._h, _p(out))
        return {"ke": out[0], "div_l2": out[1], "div_max": out[2]}

    def compute_forces(self) -> np.ndarray:
        """ComputeForces' 22 sums, Pthrust, Pdrag, EffPDef, EffPDefBnd and the grid mass
        (source/operators/FluidSolidForces.cpp:17-222, source/obstacles/Obstacle.cpp:266-295)."""
        out = np.zeros(27, dtype=np.float64)
        lib().orc_compute_forces(self._h, _p(out))
        return out

    def dissipation(self) -> np.ndarray:
        """ComputeDissipation's 20 sums (source/operators/ComputeDissipation.cpp:119-160 order)."""
        out = np.zeros(20, dtype=np.float64)
        lib().orc_dissipation(self._h, _p(out))
        return out


def poisson_solve(rhs: np.ndarray, h: float) -> np.ndarray:
    """PoissonSolverPeriodic on an h^3-premultiplied RHS (shape (nz,ny,nx))."""
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    nz, ny, nx = rhs.shape
    p = np.empty_like(rhs)
    if lib().orc_poisson_solve_field(nx, ny, nz, h, _p(rhs), _p(p)) != 0:
        raise ValueError("oracle: sizes must be powers of two")
    return p


def lab_shift(f: np.ndarray, g: int, dx: int, dy: int, dz: int) -> np.ndarray:
    f = np.ascontiguousarray(f, dtype=np.float64)
    nz, ny, nx = f.shape
    out = np.empty_like(f)
    if lib().orc_lab_shift(_p(f), _p(out), nx, ny, nz, g, dx, dy, dz) != 0:
        raise ValueError("oracle: bad lab shift arguments")
    return out


def set_num_threads(n: int):
    lib().orc_set_num_threads(n)


def num_threads() -> int:
    return lib().orc_num_threads()


def spectral(u: np.ndarray, v: np.ndarray, w: np.ndarray, h: float, nu: float, band: bool = False):
    """SpectralManipFFTW::_compute_analysis and _compute_largeModesForcing
    (source/spectralOperators/SpectralManipFFTW.cpp:25-193) restated with numpy's r2c
    DFT (the transform FFTW computes; FFTW 3.3.7 is not vendored) on [z][y][x]
    arrays. The reference halves its fastest axis (z in its x-slowest buffer);
    here the halved axis is x (the last): the sums run over the same
    conjugate-symmetric spectrum with the same multiplicities.
    Returns (stats, E_msr, band-filtered c2r fields or None): stats as
    HITstatistics (tke, eps, uprime, lambda, Re_lambda, l_integral,
    tau_integral, tke_filtered)."""
    nz, ny, nx = u.shape
    N = nx * ny * nz  # normalizeFFT
    U, V, W = (np.fft.rfftn(f) for f in (u, v, w))
    ii = np.arange(nx // 2 + 1)[None, None, :]
    jj = np.where(np.arange(ny) <= ny // 2, np.arange(ny), np.arange(ny) - ny)[None, :, None]
    kk = np.where(np.arange(nz) <= nz // 2, np.arange(nz), np.arange(nz) - nz)[:, None, None]
    wfx, wfy, wfz = (2 * np.pi / (n * h) for n in (nx, ny, nz))
    mult = np.where((ii == 0) | (ii == nx // 2), 1.0, 2.0)
    kx, ky, kz = ii * wfx, jj * wfy, kk * wfz
    k2 = kx * kx + ky * ky + kz * kz
    dX = 2 * np.sin(2 * np.pi / nx * ii)
    dY = 2 * np.sin(2 * np.pi / ny * jj)
    dZ = 2 * np.sin(2 * np.pi / nz * kk)
    OX = 1j * (dY * W - dZ * V)
    OY = 1j * (dZ * U - dX * W)
    OZ = 1j * (dX * V - dY * U)
    E = mult / 2 * (np.abs(U) ** 2 + np.abs(V) ** 2 + np.abs(W) ** 2)
    tke = E.sum()
    eps = (mult / 2 * (np.abs(OX) ** 2 + np.abs(OY) ** 2 + np.abs(OZ) ** 2)).sum()
    with np.errstate(divide="ignore", invalid="ignore"):
        lint = np.where(k2 > 0, E / np.sqrt(np.where(k2 > 0, k2, 1.0)), 0.0).sum()
    nmax = max(nx, ny, nz)
    nyq = nmax // 2
    nbin = nyq - 1
    kind = ii * ii + jj * jj + kk * kk
    sel = np.broadcast_to(kind < nyq * nyq, E.shape)
    bins = np.floor(np.sqrt(np.broadcast_to(kind, E.shape)[sel]) * ((nyq - 1) / nyq)).astype(np.int64)
    E_msr = np.bincount(bins, weights=E[sel], minlength=nbin)[:nbin] / N ** 2
    st = {"tke": tke / N ** 2, "eps": eps * 2 * nu / (N * 2 * h) ** 2}
    st["uprime"] = np.sqrt(2 * st["tke"] / 3)
    st["lambda"] = np.sqrt(15 * nu / st["eps"]) * st["uprime"]
    st["Re_lambda"] = st["uprime"] * st["lambda"] / nu
    st["l_integral"] = lint / tke
    st["tau_integral"] = st["l_integral"] / st["uprime"]
    filtered = None
    if band:
        keep = np.broadcast_to((k2 > 0) & (k2 <= 4), E.shape)
        st["tke_filtered"] = E[keep].sum() / N ** 2
        # FFTW's c2r is unnormalised: N times numpy's irfftn
        filtered = tuple(N * np.fft.irfftn(np.where(keep, F, 0), s=u.shape, axes=(0, 1, 2)) for F in (U, V, W))
    return st, E_msr, filtered


def spectral_forcing(u, v, w, h, nu, dt, target_tke=0.0, injection_rate=0.0, prev_tke=0.0):
    """SpectralForcing::operator() (source/spectralOperators/SpectralForcing.cpp:23-86)
    on FP64 arrays: returns the forced (u, v, w) and (totalKinEn, largeModesKinEn,
    viscousDissip, totalDissipRate, injectionRate, next totalKinEnPrev)."""
    st, _, filt = spectral(u, v, w, h, nu, band=True)
    N = u.size
    tke, tkeF = st["tke"], st["tke_filtered"]
    rate = 0.0
    if target_tke > 0:
        rate = (target_tke - tke) / dt
    elif injection_rate > 0:
        rate = injection_rate
    fac = dt * rate / (2 * tkeF)
    out = (u, v, w)
    prev = tke
    if fac > 0:
        prev = tke + dt * rate
        out = tuple(f + fac / N * g for f, g in zip((u, v, w), filt))
    return out, (tke, tkeF, st["eps"], (prev_tke - tke) / dt, rate, prev)

