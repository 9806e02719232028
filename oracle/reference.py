"""ORACLE CHECKER — test infrastructure only.

ctypes binding of ``oracle/_ref/libref.so``: the reference's own operator
sources (source/operators/AdvectionDiffusion.cpp, PressureRHS.cpp,
PressureProjection.cpp, source/poisson/PoissonSolverPeriodic.cpp,
PoissonSolver.cpp) compiled unmodified against the stand-ins in
``oracle/ref_shim`` (``make -C oracle ref``; needs the reference tree, which
only the build machine has). It runs the reference's operator() objects on a
one-process grid of FluidBlocks, so the oracle's restatement can be checked
against the reference's arithmetic. The FFT inside PoissonSolverPeriodic is
the stand-in's direct DFT (FFTW is not in the reference snapshot); everything
else on the path is the reference's code. Only tests import this module.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref.so")
REFERENCE_SOURCE = os.environ.get("CUP_REFERENCE_SOURCE", "/root/reference/source")
FIELDS = {"u": 0, "v": 1, "w": 2, "p": 3, "chi": 4, "tmpU": 5, "tmpV": 6, "tmpW": 7}
_lib = None


def available() -> bool:
    """The library is built, or can be (the reference tree is present)."""
    return os.path.exists(LIB_PATH) or os.path.isdir(REFERENCE_SOURCE)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REFERENCE={REFERENCE_SOURCE}"], check=True)
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.ref_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, dp, C.c_double, C.c_int]
        L.ref_create.restype = C.c_void_p
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_set_field.argtypes = [C.c_void_p, C.c_int, dp]
        L.ref_get_field.argtypes = [C.c_void_p, C.c_int, dp]
        L.ref_get_rhs.argtypes = [C.c_void_p, dp]
        L.ref_operator.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
        L.ref_operator.restype = C.c_int
        ip = C.POINTER(C.c_int)
        L.ref_add_sphere.argtypes = [C.c_void_p, C.c_double, dp, dp, ip, ip]
        L.ref_add_sphere.restype = C.c_int
        L.ref_obstacle.argtypes = [C.c_void_p, dp]
        L.ref_obstacle.restype = C.c_int
        L.ref_set_clock.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.ref_flush_logs.argtypes = []
        # the reference's logger writes its files (forceValues_0.dat, ...) once
        # more when the library unloads, after the interpreter's exit handlers:
        # into a scratch directory, not wherever the process happens to be
        atexit.register(os.chdir, tempfile.mkdtemp(prefix="cup_ref_logs_"))
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def flush_logs():
    """Writes the reference's buffered log files into the working directory."""
    lib().ref_flush_logs()


class ReferenceSim:
    """The reference's periodic pipeline objects (SimulationData, FluidGridMPI,
    ObstacleVector, CreateObstacles, AdvectionDiffusion, PressureRHS,
    PressureProjection, UpdateObstacles, Penalization, ComputeForces) on an
    nx x ny x nz grid."""

    PIPELINE = ("CreateObstacles", "AdvectionDiffusion", "PressureRHS", "PressureProjection", "UpdateObstacles",
                "Penalization", "ComputeForces")

    def __init__(self, nx, ny, nz, maxextent, nu, uinf=(0.0, 0.0, 0.0), lambda_=1e6, implicit=True):
        ui = np.ascontiguousarray(uinf, dtype=np.float64)
        self.shape = (nz, ny, nx)
        self.step, self.time = 0, 0.0
        self._h = lib().ref_create(nx, ny, nz, maxextent, nu, _p(ui), lambda_, int(bool(implicit)))
        if not self._h:
            raise RuntimeError("reference: construction failed (see stderr)")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ref_destroy(self._h)
            self._h = None

    def set(self, name: str, f):
        a = np.ascontiguousarray(f, dtype=np.float64)
        assert a.shape == self.shape
        lib().ref_set_field(self._h, FIELDS[name], _p(a))

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        lib().ref_get_field(self._h, FIELDS[name], _p(out))
        return out

    def set_velocity(self, u, v, w):
        for n, f in zip("uvw", (u, v, w)):
            self.set(n, f)

    def velocity(self):
        return self.get("u"), self.get("v"), self.get("w")

    def rhs(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        lib().ref_get_rhs(self._h, _p(out))
        return out

    def add_sphere(self, radius, position, velocity, forced=(1, 1, 1), fix_frame=(0, 0, 0)):
        pos = np.ascontiguousarray(position, dtype=np.float64)
        vel = np.ascontiguousarray(velocity, dtype=np.float64)
        f = (C.c_int * 3)(*[int(bool(x)) for x in forced])
        ff = (C.c_int * 3)(*[int(bool(x)) for x in fix_frame])
        if lib().ref_add_sphere(self._h, radius, _p(pos), _p(vel), f, ff):
            raise RuntimeError("reference: adding the sphere failed (see stderr)")

    def obstacle(self) -> dict:
        out = np.zeros(48, dtype=np.float64)
        if lib().ref_obstacle(self._h, _p(out)):
            raise RuntimeError("reference: no obstacle")
        return {"force": out[0:3], "torque": out[3:6], "com": out[6:9], "transVel": out[9:12],
                "angVel": out[12:15], "position": out[15:18], "uinf": out[18:21], "mass": out[21],
                "forces": out[22:48]}

    def timestep(self, dt: float):
        """Simulation::timestep (source/Simulation.cpp:593-623) over the pipeline."""
        lib().ref_set_clock(self._h, self.step, self.time, dt)
        for name in self.PIPELINE:
            self.operator(name, dt)
        self.step += 1
        self.time += dt

    def operator(self, name: str, dt: float):
        rc = lib().ref_operator(self._h, name.encode(), dt)
        if rc:
            raise RuntimeError(f"reference operator {name} failed ({rc})")
