"""Python host side mirroring CubismUP_3D's pybind11 API for the periodic hot path.

Reference interface (source/bindings/Simulation.cpp:59-94, source/bindings/Obstacles.cpp:79-129):
``SimulationData(comm, CFL, cells, uinf)``, ``Simulation(SimulationData)`` with
``run()`` and ``add_obstacle(Sphere(...))``; operators are the pipeline entries
of ``Simulation::setupOperators`` (source/Simulation.cpp:307-401) driven by
``operator()(double dt)`` with ``getName()``. Every call goes through the C ABI
of ``libcup_b200.so`` (include/cup_b200.h); arguments the reference rejects
with ``std::invalid_argument`` raise ``ValueError`` here as pybind11 would.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L

PERIODIC = "periodic"
BLOCK_SIZE = 16  # CUP_BLOCK_SIZE (source/Definitions.h:27-29)


@dataclass
class SimulationData:
    """Hot-path subset of SimulationData (source/SimulationData.h:46-179).

    Struct defaults follow the reference's struct (not its CLI defaults):
    ``DLM = 1`` (lambda = 1/dt, SimulationData.h:98), ``rampup = 100``
    (SimulationData.h:143). Only periodic boundaries are supported.
    """

    CFL: float = 0.1
    cells: Tuple[int, int, int] = (64, 64, 64)
    uinf: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    comm: object = None
    nu: float = 0.0
    lambda_: float = -1.0
    DLM: float = 1.0
    rampup: int = 100
    nsteps: int = 0
    endTime: float = 0.0
    extent: float = 1.0  # maxextent: h = extent / max(cells)
    bImplicitPenalization: bool = False
    BCx_flag: str = PERIODIC
    BCy_flag: str = PERIODIC
    BCz_flag: str = PERIODIC
    precision: str = "fp64"  # "fp64" | "fp32_dc"
    scheme: str = "ref"      # "ref" | "upwind3_rk2"
    dc_tol: float = 1e-10
    dc_max_iter: int = 2
    dc_min_iter: int = 1
    device: int = 0
    z_halo: int = 0           # > 0: one rank's z-slab with this many ghost planes a side (slab.SlabSimulation)
    verbose: bool = False
    freqDiagnostics: int = 0  # ComputeDissipation every this many steps (0: off), to diagnostics.dat
    turbKinEn_target: float = 0.0   # SpectralForcing: hold the kinetic energy at this value ...
    enInjectionRate: float = 0.0    # ... or inject energy at this rate (SimulationData.cpp:60-66)
    saveFreq: int = 0         # restart dumps every this many steps (0: off)
    saveTime: float = 0.0     # ... or every this much simulated time (0: off)
    path4serialization: str = "./"

    def __post_init__(self):
        self.setCells(*self.cells)

    def setCells(self, nx: int, ny: int, nz: int):
        """SimulationData::setCells (source/SimulationData.cpp:280-291)."""
        if nx % BLOCK_SIZE or ny % BLOCK_SIZE or nz % BLOCK_SIZE:
            raise ValueError("Number of cells must be multiple of block size * number of processes.")
        self.cells = (int(nx), int(ny), int(nz))

    @property
    def bpd(self) -> Tuple[int, int, int]:
        return tuple(c // BLOCK_SIZE for c in self.cells)

    def to_config(self) -> L.CupConfig:
        if (self.BCx_flag, self.BCy_flag, self.BCz_flag) != (PERIODIC,) * 3:
            raise ValueError("only periodic boundaries are supported (bUseFourierBC)")
        if self.lambda_ <= 0 and self.DLM <= 0:
            raise ValueError("need lambda > 0 or DLM > 0 (SimulationData.cpp:203)")
        cfg = L.CupConfig()
        cfg.bpdx, cfg.bpdy, cfg.bpdz = self.bpd
        cfg.maxextent = float(self.extent)
        cfg.nu = float(self.nu)
        cfg.CFL = float(self.CFL)
        cfg.lambda_ = float(self.lambda_)
        cfg.DLM = float(self.DLM)
        cfg.uinf[:] = [float(x) for x in self.uinf]
        cfg.rampup = int(self.rampup)
        cfg.bImplicitPenalization = int(bool(self.bImplicitPenalization))
        cfg.precision = {"fp64": L.CUP_PREC_FP64, "fp32_dc": L.CUP_PREC_FP32_DC}[self.precision]
        cfg.scheme = {"ref": L.CUP_SCHEME_REF, "upwind3_rk2": L.CUP_SCHEME_UPWIND3_RK2}[self.scheme]
        cfg.dc_tol = float(self.dc_tol)
        cfg.dc_max_iter = int(self.dc_max_iter)
        cfg.dc_min_iter = int(self.dc_min_iter)
        cfg.device = int(self.device)
        cfg.z_halo = int(self.z_halo)
        return cfg


@dataclass
class ObstacleArguments:
    """ObstacleArguments (source/obstacles/Obstacle.h:60-75)."""

    length: float = 0.0
    position: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    quaternion: Tuple[float, float, float, float] = (1.0, 0.0, 0.0, 0.0)
    enforcedVelocity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    bForcedInSimFrame: Tuple[bool, bool, bool] = (False, False, False)
    bFixFrameOfRef: Tuple[bool, bool, bool] = (False, False, False)
    bFixToPlanar: bool = False
    bComputeForces: bool = True


class Sphere(ObstacleArguments):
    """ObstacleAndSphereArguments constructor of the bindings
    (source/bindings/Obstacles.cpp:57-82): ``Sphere(radius, umax, tmax,
    accel_decel, bHemi, **kwargs)`` with ObstacleArguments as kwargs."""

    def __init__(self, radius: float = -1.0, umax: float = 0.0, tmax: float = 1.0,
                 accel_decel: bool = False, bHemi: bool = False, **kwargs):
        length = float(kwargs.pop("length", 0.0))
        if radius > 0 and length > 0 and radius != 0.5 * length:
            raise ValueError("Cannot specify both `radius` and `length`.")
        elif radius <= 0 and length <= 0:
            raise ValueError("Expected a `radius` or `length`.")
        elif radius > 0:
            length = 2.0 * radius
        else:
            radius = 0.5 * length
        super().__init__(length=length)
        for k in ("position", "quaternion", "enforcedVelocity", "bForcedInSimFrame", "bFixFrameOfRef",
                  "bFixToPlanar", "bComputeForces"):
            if k in kwargs:
                setattr(self, k, kwargs.pop(k))
        if kwargs:
            raise ValueError(f"unknown Sphere arguments: {sorted(kwargs)}")
        if accel_decel or bHemi:
            raise ValueError("accel_decel and hemisphere spheres are not supported")
        self.radius = float(radius)
        self.umax, self.tmax = umax, tmax
        self.accel_decel, self.bHemi = accel_decel, bHemi

    def to_struct(self) -> L.CupSphere:
        s = L.CupSphere()
        s.radius = self.radius
        s.position[:] = [float(x) for x in self.position]
        s.enforcedVelocity[:] = [float(x) for x in self.enforcedVelocity]
        s.bForcedInSimFrame[:] = [int(bool(x)) for x in self.bForcedInSimFrame]
        s.bFixFrameOfRef[:] = [int(bool(x)) for x in self.bFixFrameOfRef]
        return s


def _as_host_f64(a, shape) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if arr.shape != shape:
        raise ValueError(f"expected an array of shape {shape} (nz, ny, nx), got {arr.shape}")
    return arr


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


_CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


def _is_torch_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


class Operator:
    """Operator (source/operators/Operator.h:16-177): ``op(dt)``, ``getName()``."""

    name = "Operator"

    def __init__(self, sim: "Simulation"):
        self.sim = sim

    def getName(self) -> str:
        return self.name

    def __call__(self, dt: float):  # pragma: no cover - abstract
        raise NotImplementedError


class CreateObstacles(Operator):
    """CreateObstacles (source/operators/ObstaclesCreate.cpp:444-540): moves a
    sphere that is not at rest in the frame by dt (transVel + uinf) and
    rebuilds its chi; nothing otherwise."""
    name = "CreateObstacles"

    def __call__(self, dt: float):
        L.check(L.lib().cup_create_obstacles(self.sim._h, float(dt)), self.sim._h, self.name)


class AdvectionDiffusion(Operator):
    name = "AdvectionDiffusion"

    def __call__(self, dt: float):
        L.check(L.lib().cup_advect_diffuse(self.sim._h, float(dt)), self.sim._h, self.name)


class PressureRHS(Operator):
    name = "PressureRHS"

    def __call__(self, dt: float):
        L.check(L.lib().cup_pressure_rhs(self.sim._h, float(dt)), self.sim._h, self.name)


class PressureProjection(Operator):
    name = "PressureProjection"

    def __call__(self, dt: float):
        st = L.CupSolveStats()
        L.check(L.lib().cup_pressure_projection(self.sim._h, float(dt), C.byref(st)), self.sim._h, self.name)
        self.last_stats = st


class UpdateObstacles(Operator):
    """UpdateObstacles (source/operators/ObstaclesUpdate.cpp:202-236): for a
    sphere with free dofs, the fluid momentum integrals and the 6x6 momentum
    balance of Obstacle::computeVelocities (source/obstacles/Obstacle.cpp:153-264)
    give the free dofs' velocities (cup_update_obstacles); forced dofs keep
    their imposed velocity."""
    name = "UpdateObstacles"

    def __call__(self, dt: float):
        L.check(L.lib().cup_update_obstacles(self.sim._h, float(dt)), self.sim._h, self.name)


class Penalization(Operator):
    name = "Penalization"

    def __call__(self, dt: float):
        ft = (C.c_double * 6)()
        L.check(L.lib().cup_penalize(self.sim._h, float(dt), ft), self.sim._h, self.name)
        self.force_torque = np.array(ft[:])


# diagnostics.dat columns of ComputeDissipation (source/operators/ComputeDissipation.cpp:162-176),
# header spelled as the reference writes it
DISSIPATION_NAMES = ("circ_x", "circ_y", "circ_z", "linImp_x", "linImp_y", "linImp_z", "linMom_x", "linMom_y",
                     "linMom_z", "angImp_x", "angImp_y", "angImp_z", "angMom_x", "angMom_y", "angMom_z", "presPow",
                     "viscPow", "helicity", "kineticEn", "enstrophy")
DIAGNOSTICS_HEADER = ("step_id time circ_x circ_y circ_y linImp_x linImp_y linImp_z linMom_x linMom_y linMom_z "
                      "angImp_x angImp_y angImp_z angMom_x angMom_y angMom_z presPow viscPow helicity kineticEn "
                      "enstrophy")


class ComputeDissipation(Operator):
    """ComputeDissipation (source/operators/ComputeDissipation.cpp:119-177): every
    ``freqDiagnostics`` steps, the 20 sums of the current fields appended to
    ``diagnostics.dat`` (header at step 0)."""
    name = "ComputeDissipation"

    def __call__(self, dt: float):
        self.sim._diagnostics_line(self.sim.step, self.sim.time)


# ComputeForces outputs (source/obstacles/Obstacle.cpp:266-295): the 22 sums in
# ObstacleBlock::sumQoI order (source/ObstacleBlock.h:81-93), the derived
# powers and efficiencies, the grid mass of chi
FORCE_NAMES = ("surfForce_x", "surfForce_y", "surfForce_z", "presForce_x", "presForce_y", "presForce_z",
               "viscForce_x", "viscForce_y", "viscForce_z", "surfTorque_x", "surfTorque_y", "surfTorque_z",
               "gamma_x", "gamma_y", "gamma_z", "drag", "thrust", "Pout", "PoutBnd", "defPower", "defPowerBnd",
               "pLocom", "Pthrust", "Pdrag", "EffPDef", "EffPDefBnd", "mass")


class ComputeForces(Operator):
    """ComputeForces (source/operators/FluidSolidForces.cpp:200-222) after
    Penalization: the surface forces of the sphere on the final velocity and
    pressure, appended to forceValues_surface_<id>.dat and
    powerValues_surface_<id>.dat in the reference's format
    (source/obstacles/Obstacle.cpp:518-556); nothing without obstacles."""
    name = "ComputeForces"

    def __call__(self, dt: float):
        if not self.sim.obstacles:
            return
        self.forces = self.sim.compute_forces()
        self.sim._forces_lines(self.sim.step, self.sim.time, self.forces)


class SpectralForcing(Operator):
    """SpectralForcing (source/spectralOperators/SpectralForcing.cpp:23-86): raises the
    energy of the band 0 < k^2 <= 4 to meet turbKinEn_target or enInjectionRate."""
    name = "SpectralForcing"

    def __call__(self, dt: float):
        st = (C.c_double * 6)()
        L.check(L.lib().cup_spectral_forcing(self.sim._h, float(dt), st), self.sim._h, self.name)
        self.stats = dict(zip(FORCING_NAMES, st[:]))


FORCING_NAMES = ("totalKinEn", "largeModesKinEn", "viscousDissip", "totalDissipRate", "injectionRate", "lIntegral")
SPECTRAL_NAMES = ("tke", "eps", "uprime", "lambda", "Re_lambda", "l_integral", "tau_integral")


class _DeviceArray:
    """A raw FP64 device allocation described by the CUDA array interface, so
    that torch.as_tensor can view it without a copy."""

    def __init__(self, ptr: int, shape, device: int):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}
        self.device = device


class PoissonSolverPeriodic:
    """PoissonSolverPeriodic (source/poisson/PoissonSolverPeriodic.cpp) bound
    to a simulation's device buffers: ``solve()`` runs the FFT chain.

    The buffer contract of PoissonSolver (source/poisson/PoissonSolver.h:51-122):
    ``data`` is the FP64 device array the RHS is written into (a torch CUDA
    tensor of shape (nz, ny, nx) viewing it without a copy), with ``stridex``,
    ``stridey``, ``stridez`` (elements) and ``data_size``; ``_offset(info)`` /
    ``_offset_ext(info)`` give a block's first cell, ``_dest`` a cell of it.
    ``reset()`` zeroes the buffer. ``solve()`` includes ``_fftw2cub`` (the
    solution goes to the pressure), so ``_fftw2cub()`` itself has nothing left
    to do."""

    def __init__(self, sim: "Simulation"):
        self.sim = sim
        ptr = C.c_void_p()
        strides = (C.c_size_t * 3)()
        size = C.c_size_t()
        L.check(L.lib().cup_poisson_buffer(sim._h, C.byref(ptr), strides, C.byref(size)), sim._h, "poisson buffer")
        self._ptr = ptr.value
        self.stridex, self.stridey, self.stridez = (int(x) for x in strides)
        self.data_size = int(size.value)

    @property
    def data(self):
        import torch
        return torch.as_tensor(_DeviceArray(self._ptr, self.sim.shape, self.sim.sd.device),
                               device=f"cuda:{self.sim.sd.device}")

    def _offset(self, info) -> int:
        """First cell of a block: ``info`` has ``index`` (bx, by, bz) or is that triple."""
        bx, by, bz = info if isinstance(info, (tuple, list)) else info.index
        return BLOCK_SIZE * (self.stridez * bz + self.stridey * by + self.stridex * bx)

    _offset_ext = _offset

    def _dest(self, offset: int, z: int, y: int, x: int) -> int:
        return offset + self.stridez * z + self.stridey * y + self.stridex * x

    def reset(self):
        L.check(L.lib().cup_poisson_reset(self.sim._h), self.sim._h, "PoissonSolver::reset")

    def _cub2fftw(self):
        """Nothing to do: the RHS is written into ``data`` directly."""

    def _fftw2cub(self):
        """Nothing to do: ``solve()`` writes the solution into the pressure."""

    def solve(self):
        st = L.CupSolveStats()
        L.check(L.lib().cup_poisson_solve(self.sim._h, C.byref(st)), self.sim._h, "PoissonSolverPeriodic")
        return st

    def solve_field(self, rhs) -> np.ndarray:
        """Solves L_2h p = rhs / h^3 for an h^3-premultiplied rhs (nz, ny, nx)."""
        r = _as_host_f64(rhs, self.sim.shape)
        p = np.empty_like(r)
        L.check(L.lib().cup_poisson_solve_field(self.sim._h, _ptr(r), _ptr(p), L.CUP_WHERE_HOST), self.sim._h)
        return p


@dataclass
class StepStats:
    dt: float
    time: float
    step: int
    umax: float
    kinetic_energy: float
    force: np.ndarray
    torque: np.ndarray
    n_solves: int
    rel_residual: float
    n_unconverged: int = 0
    n_solves_total: int = 0

    @classmethod
    def from_c(cls, s: L.CupStepStats) -> "StepStats":
        return cls(s.dt, s.time, s.step, s.umax, s.kinetic_energy, np.array(s.force[:]), np.array(s.torque[:]),
                   s.n_solves, s.rel_residual, s.n_unconverged, s.n_solves_total)


class Simulation:
    """Simulation (source/Simulation.cpp): owns one device handle."""

    def __init__(self, sd: SimulationData):
        self.sd = sd
        cfg = sd.to_config()
        h = C.c_void_p()
        rc = L.lib().cup_create(C.byref(cfg), C.byref(h))
        if rc != L.CUP_OK:
            L.check(rc, None, "cup_create (see stderr for the reason)")
        self._h = h
        cells = (C.c_int * 3)()
        hg = C.c_double()
        L.lib().cup_get_dims(self._h, cells, C.byref(hg))
        self.cells = tuple(cells[:])
        self.h = hg.value
        self.shape = (self.cells[2], self.cells[1], self.cells[0])
        self.obstacles: List[Sphere] = []
        self.pressureSolver = PoissonSolverPeriodic(self)
        # pipeline of the periodic hot path in the order of
        # Simulation::setupOperators (source/Simulation.cpp:307-401)
        self.pipeline: List[Operator] = [CreateObstacles(self), AdvectionDiffusion(self), PressureRHS(self),
                                         PressureProjection(self), UpdateObstacles(self), Penalization(self),
                                         ComputeForces(self), ComputeDissipation(self)]
        if sd.turbKinEn_target > 0 and sd.enInjectionRate > 0:
            raise ValueError("give either turbKinEn_target or enInjectionRate, not both (SimulationData.cpp:64-66)")
        self.forcing = sd.turbKinEn_target > 0 or sd.enInjectionRate > 0
        if self.forcing:
            L.check(L.lib().cup_set_spectral_forcing(h, float(sd.turbKinEn_target), float(sd.enInjectionRate)), h,
                    "spectral forcing")
            self.pipeline.insert(2, SpectralForcing(self))
        self.step = 0
        self.time = 0.0
        self.dt = 0.0

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            L.lib().cup_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def sim(self) -> SimulationData:
        return self.sd

    def set_stream(self, stream_ptr: Optional[int]):
        """Runs the handle's work on the CUDA stream ``stream_ptr`` (None: the
        handle's own stream)."""
        L.check(L.lib().cup_set_stream(self._h, C.c_void_p(stream_ptr or 0)), self._h, "set_stream")
        self._bound_stream = stream_ptr or None

    def bind_torch_stream(self):
        """Runs the handle's work on torch's current stream of its device, so that
        torch tensors passed by pointer are ordered with it. torch reports the
        legacy default stream as 0; the runtime's name for it is cudaStreamLegacy."""
        import torch
        ptr = torch.cuda.current_stream(self.sd.device).cuda_stream or _CUDA_STREAM_LEGACY
        if getattr(self, "_bound_stream", None) != ptr:
            self.set_stream(ptr)

    def sync(self):
        L.check(L.lib().cup_sync(self._h), self._h, "sync")

    # -- obstacles -------------------------------------------------------------
    def add_obstacle(self, obstacle):
        if not isinstance(obstacle, Sphere):
            raise ValueError(str(obstacle))
        s = obstacle.to_struct()
        L.check(L.lib().cup_add_sphere(self._h, C.byref(s)), self._h, "add_obstacle")
        self.obstacles.append(obstacle)

    def obstacle_state(self) -> dict:
        f, t, c, u = (C.c_double * 3)(), (C.c_double * 3)(), (C.c_double * 3)(), (C.c_double * 3)()
        L.check(L.lib().cup_get_obstacle_state(self._h, f, t, c, u), self._h, "obstacle_state")
        tv, av, q = (C.c_double * 3)(), (C.c_double * 3)(), (C.c_double * 4)()
        L.check(L.lib().cup_get_sphere_motion(self._h, tv, av, q), self._h, "obstacle_state")
        return {"force": np.array(f[:]), "torque": np.array(t[:]), "com": np.array(c[:]), "uinf": np.array(u[:]),
                "transVel": np.array(tv[:]), "angVel": np.array(av[:]), "quaternion": np.array(q[:])}

    def set_sphere_motion(self, transVel, angVel, quaternion=(1.0, 0.0, 0.0, 0.0)):
        """Restores the sphere's velocities and orientation (Obstacle::restart)."""
        tv, av = (C.c_double * 3)(*map(float, transVel)), (C.c_double * 3)(*map(float, angVel))
        q = (C.c_double * 4)(*map(float, quaternion))
        L.check(L.lib().cup_set_sphere_motion(self._h, tv, av, q), self._h, "set_sphere_motion")

    # -- fields ----------------------------------------------------------------
    def set_velocity(self, u, v, w):
        if all(_is_torch_cuda(a) for a in (u, v, w)):
            import torch
            ts = [a.detach().to(torch.float64).contiguous() for a in (u, v, w)]
            for t in ts:
                if tuple(t.shape) != self.shape:
                    raise ValueError(f"expected shape {self.shape}")
            torch.cuda.current_stream().synchronize()
            L.check(L.lib().cup_set_velocity(self._h, *[C.c_void_p(t.data_ptr()) for t in ts], L.CUP_WHERE_DEVICE),
                    self._h, "set_velocity")
            self.sync()
            return
        arrs = [_as_host_f64(a if not hasattr(a, "numpy") else a.detach().cpu().numpy(), self.shape) for a in (u, v, w)]
        L.check(L.lib().cup_set_velocity(self._h, *[_ptr(a) for a in arrs], L.CUP_WHERE_HOST), self._h, "set_velocity")

    def velocity(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        out = [np.empty(self.shape, dtype=np.float64) for _ in range(3)]
        L.check(L.lib().cup_get_velocity(self._h, *[_ptr(a) for a in out], L.CUP_WHERE_HOST), self._h, "velocity")
        return tuple(out)

    def velocity_into(self, u, v, w):
        """Copies the velocity into three FP64 CUDA torch tensors (device to device)."""
        self.bind_torch_stream()
        L.check(L.lib().cup_get_velocity(self._h, C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                         C.c_void_p(w.data_ptr()), L.CUP_WHERE_DEVICE), self._h, "velocity_into")

    # -- raw device fields and the discrete adjoint (torch CUDA tensors) ---------
    @property
    def storage_dtype(self):
        """torch dtype of the device fields: float64 (fp64) or float32 (fp32_dc)."""
        import torch
        return torch.float32 if self.sd.precision == "fp32_dc" else torch.float64

    def _check_raw(self, t, what):
        if not _is_torch_cuda(t) or t.dtype != self.storage_dtype or not t.is_contiguous() or \
                tuple(t.shape) != (3,) + self.shape:
            raise ValueError(f"{what}: expected a contiguous CUDA tensor of shape {(3,) + self.shape} "
                             f"and dtype {self.storage_dtype}")

    def velocity_raw(self, out=None):
        """The velocity as one (3, nz, ny, nx) CUDA tensor in the storage dtype,
        copied on the handle's stream."""
        import torch
        if out is None:
            out = torch.empty((3,) + self.shape, dtype=self.storage_dtype, device=f"cuda:{self.sd.device}")
        self._check_raw(out, "velocity_raw")
        self.bind_torch_stream()
        L.check(L.lib().cup_get_velocity_raw(self._h, *[C.c_void_p(out[i].data_ptr()) for i in range(3)]),
                self._h, "velocity_raw")
        return out

    def set_velocity_raw(self, t):
        """Sets the velocity from a (3, nz, ny, nx) CUDA tensor in the storage dtype."""
        self._check_raw(t, "set_velocity_raw")
        self.bind_torch_stream()
        L.check(L.lib().cup_set_velocity_raw(self._h, *[C.c_void_p(t[i].data_ptr()) for i in range(3)]),
                self._h, "set_velocity_raw")

    def adjoint_step(self, state, dt: float, lam):
        """Discrete adjoint of ``timestep(dt)`` taken from ``state``: ``lam``
        (dJ/du after the step, (3, nz, ny, nx)) becomes dJ/du before it, in place."""
        self._check_raw(state, "adjoint_step state")
        self._check_raw(lam, "adjoint_step lam")
        self.bind_torch_stream()
        L.check(L.lib().cup_adjoint_step(self._h, *[C.c_void_p(state[i].data_ptr()) for i in range(3)], float(dt),
                                         *[C.c_void_p(lam[i].data_ptr()) for i in range(3)]), self._h, "adjoint_step")

    def adjoint_step_obstacle(self, state, dt: float, lam, w_force, g_chi, g_vel):
        """Discrete adjoint of ``timestep(dt)`` of a handle with the sphere, taken
        from ``state``, for J = <g, u_T> + sum over steps of w_force . F (F the
        penalization force): ``lam`` becomes dJ/du before the step (in place);
        dJ/dchi is added to ``g_chi`` (FP64 CUDA tensor of the grid's shape) and
        dJ/dU for the sphere's target velocity (uinf fixed) to ``g_vel`` (3 FP64)."""
        import torch
        self._check_raw(state, "adjoint_step_obstacle state")
        self._check_raw(lam, "adjoint_step_obstacle lam")
        for t, shape, what in ((g_chi, self.shape, "g_chi"), (g_vel, (3,), "g_vel")):
            if not _is_torch_cuda(t) or t.dtype != torch.float64 or not t.is_contiguous() or tuple(t.shape) != shape:
                raise ValueError(f"adjoint_step_obstacle: {what} must be a contiguous FP64 CUDA tensor of shape {shape}")
        self.bind_torch_stream()
        w = (C.c_double * 3)(*[float(x) for x in w_force])
        L.check(L.lib().cup_adjoint_step_obstacle(self._h, *[C.c_void_p(state[i].data_ptr()) for i in range(3)],
                                                  float(dt), *[C.c_void_p(lam[i].data_ptr()) for i in range(3)], w,
                                                  C.c_void_p(g_chi.data_ptr()), C.c_void_p(g_vel.data_ptr())),
                self._h, "adjoint_step_obstacle")

    def set_chi(self, chi):
        """Replaces the obstacle's characteristic function (host array of the
        grid's shape; only the obstacle's active box is read by the step)."""
        a = _as_host_f64(chi, self.shape)
        L.check(L.lib().cup_set_chi(self._h, _ptr(a), L.CUP_WHERE_HOST), self._h, "set_chi")

    def set_sphere_velocity(self, vel):
        """Sets the sphere's penalization target velocity (uinf unchanged)."""
        v = (C.c_double * 3)(*[float(x) for x in vel])
        L.check(L.lib().cup_set_sphere_velocity(self._h, v), self._h, "set_sphere_velocity")

    def _get1(self, fn, what) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        L.check(fn(self._h, _ptr(out), L.CUP_WHERE_HOST), self._h, what)
        return out

    def pressure(self) -> np.ndarray:
        return self._get1(L.lib().cup_get_pressure, "pressure")

    def chi(self) -> np.ndarray:
        return self._get1(L.lib().cup_get_chi, "chi")

    def rhs(self) -> np.ndarray:
        return self._get1(L.lib().cup_get_rhs, "rhs")

    # -- driver ------------------------------------------------------------------
    def max_velocity(self) -> float:
        m = C.c_double()
        L.check(L.lib().cup_max_velocity(self._h, C.byref(m)), self._h, "max_velocity")
        return m.value

    def calcMaxTimestep(self) -> float:
        dt = C.c_double()
        L.check(L.lib().cup_calc_max_timestep(self._h, C.byref(dt)), self._h, "calcMaxTimestep")
        self.dt = dt.value
        return self.dt

    def timestep(self, dt: float, stats: bool = True) -> Optional[StepStats]:
        """Simulation::timestep (source/Simulation.cpp:593-623); returns True when finished."""
        st = L.CupStepStats()
        dump = self._maybe_serialize(dt)
        L.check(L.lib().cup_step(self._h, float(dt), C.byref(st) if stats else None), self._h, "timestep")
        if self.forcing:
            self._forcing_line(self.step, self.time, dt)
        self._diagnostics_line(self.step, self.time)
        self.step += 1
        self.time += dt
        self.dt = dt
        if dump:
            self.serialize()
        return StepStats.from_c(st) if stats else None

    def _advance(self, dt: float, stats: bool = False) -> Optional[StepStats]:
        """One cup_step with the clock update and nothing else: no restart dump,
        no diagnostics.dat or forcingData.dat line. For the adjoint rollouts,
        whose forward and checkpoint recomputation must leave the run's output
        files and restart point as they were."""
        st = L.CupStepStats()
        L.check(L.lib().cup_step(self._h, float(dt), C.byref(st) if stats else None), self._h, "timestep")
        self.step += 1
        self.time += dt
        self.dt = dt
        return StepStats.from_c(st) if stats else None

    def use_graphs(self, on: bool = True):
        """run_steps replays its steady-state steps as a captured CUDA graph (default on)."""
        L.check(L.lib().cup_set_graphs(self._h, int(bool(on))), self._h, "use_graphs")

    def prepare_run(self, nsteps: int) -> int:
        """Captures (without running) the CUDA graphs that run_steps(nsteps)
        replays from the current state; returns how many (cup_prepare_run)."""
        c = C.c_int()
        L.check(L.lib().cup_prepare_run(self._h, int(nsteps), C.byref(c)), self._h, "prepare_run")
        return c.value

    def run_steps(self, nsteps: int) -> StepStats:
        """nsteps of calcMaxTimestep + timestep with dt chained on the device."""
        st = L.CupStepStats()
        L.check(L.lib().cup_run(self._h, int(nsteps), C.byref(st)), self._h, "run")
        self.step, self.time, self.dt = st.step, st.time, st.dt
        return StepStats.from_c(st)

    def run(self) -> StepStats:
        """Simulation::run (source/Simulation.cpp:582-591): until nsteps or endTime."""
        if self.sd.nsteps <= 0 and self.sd.endTime <= 0:
            raise ValueError("set nsteps or endTime before run()")
        last = None
        if (self.sd.endTime <= 0 and self.sd.freqDiagnostics == 0 and self.sd.saveFreq == 0 and self.sd.saveTime == 0
                and not self.forcing):
            return self.run_steps(self.sd.nsteps - self.step)
        while True:
            dt = self.calcMaxTimestep()
            last = self.timestep(dt)
            if (self.sd.endTime > 0 and self.time > self.sd.endTime) or (
                    self.sd.nsteps != 0 and self.step >= self.sd.nsteps):
                return last

    def compute_forces(self) -> dict:
        """ComputeForces' surface forces of the current fields (cup_compute_forces),
        by name (FORCE_NAMES); all zero without an obstacle."""
        out = (C.c_double * 27)()
        L.check(L.lib().cup_compute_forces(self._h, out), self._h, "compute_forces")
        return dict(zip(FORCE_NAMES, out[:]))

    def _forces_lines(self, step: int, time: float, f: dict, oid: int = 0):
        """Obstacle::_writeSurfForcesToFile (source/obstacles/Obstacle.cpp:518-556):
        tab-separated, header at step 0, values in scientific notation with 8
        significant digits."""
        tab = "\t"
        e = lambda x: f"{x:.7e}"  # noqa: E731  (std::scientific, precision digits10 + 1)
        with open(f"forceValues_surface_{oid}.dat", "a") as fh:
            if step == 0:
                fh.write(tab.join(["step", "time", "mass", "force_x", "force_y", "force_z", "torque_x", "torque_y",
                                   "torque_z", "presF_x", "presF_y", "presF_z", "viscF_x", "viscF_y", "viscF_z",
                                   "gamma_x", "gamma_y", "gamma_z", "drag", "thrust"]) + "\n")
            keys = ("mass", "surfForce_x", "surfForce_y", "surfForce_z", "surfTorque_x", "surfTorque_y", "surfTorque_z",
                    "presForce_x", "presForce_y", "presForce_z", "viscForce_x", "viscForce_y", "viscForce_z",
                    "gamma_x", "gamma_y", "gamma_z", "drag", "thrust")
            fh.write(f"{step}{tab}" + tab.join([e(time)] + [e(f[k]) for k in keys]) + "\n")
        with open(f"powerValues_surface_{oid}.dat", "a") as fh:
            if step == 0:
                fh.write(tab.join(["step", "time", "Pthrust", "Pdrag", "Pout", "pDef", "etaPDef", "pLocom", "PoutBnd",
                                   "defPowerBnd", "etaPDefBnd"]) + "\n")
            vals = [time, f["Pthrust"], f["Pdrag"], f["Pout"], -f["defPower"], f["EffPDef"], f["pLocom"], f["PoutBnd"],
                    -f["defPowerBnd"], f["EffPDefBnd"]]
            fh.write(f"{step}{tab}" + tab.join(e(x) for x in vals) + "\n")

    def compute_dissipation(self) -> dict:
        """ComputeDissipation's 20 FP64 sums of the current fields, by diagnostics.dat column name."""
        out = (C.c_double * 20)()
        L.check(L.lib().cup_compute_dissipation(self._h, out), self._h, "compute_dissipation")
        return dict(zip(DISSIPATION_NAMES, out[:]))

    def _diagnostics_line(self, step: int, time: float, path: str = "diagnostics.dat"):
        f = int(self.sd.freqDiagnostics)
        if f == 0 or step % f:
            return
        d = self.compute_dissipation()
        with open(path, "a") as fh:
            if step == 0:
                fh.write(DIAGNOSTICS_HEADER + "\n")
            fh.write(" ".join([str(step), f"{time:g}"] + [f"{d[k]:g}" for k in DISSIPATION_NAMES]) + "\n")

    # -- spectral analysis -------------------------------------------------------
    def spectral_analysis(self) -> dict:
        """SpectralAnalysis (source/spectralOperators/SpectralManipFFTW.cpp:110-193): HIT
        statistics of the current velocity and its shell spectrum E_msr (key
        ``spectrum``; shell i at wavenumber (i + 1) 2 pi / L, L the largest extent)."""
        n = max(self.cells)
        nbin = n // 2 - 1
        st, spec = (C.c_double * 7)(), (C.c_double * nbin)()
        L.check(L.lib().cup_spectral_analysis(self._h, st, spec, nbin), self._h, "spectral_analysis")
        out = dict(zip(SPECTRAL_NAMES, st[:]))
        out["spectrum"] = np.array(spec[:])
        out["k"] = (np.arange(nbin) + 1) * 2 * np.pi / (n * self.h)
        return out

    def _forcing_line(self, step: int, time: float, dt: float, path: str = "forcingData.dat"):
        """The forcingData.dat line of SpectralForcing (SpectralForcing.cpp:56-69)."""
        st = (C.c_double * 6)()
        L.check(L.lib().cup_get_forcing_stats(self._h, st), self._h, "forcing stats")
        with open(path, "a") as fh:
            if step == 0:
                fh.write("step \t time \t dt \t totalKinEn \t largeModesKinEn \t viscousDissip \t "
                         "totalDissipRate \t injectionRate \t lIntegral\n")
            fh.write("\t".join([str(step)] + [f"{x:.7e}" for x in (time, dt) + tuple(st[:])]) + "\n")

    # -- restart files -----------------------------------------------------------
    def serialize(self, append: str = "") -> str:
        """Simulation::_serialize (source/Simulation.cpp:426-524): ``restart.status`` and
        ``<name>.status`` (time, stepid, uinf as the reference prints them), the
        obstacle's ``<name>_0.txt`` (Obstacle::save, source/obstacles/Obstacle.cpp:402-423)
        and the velocity, pressure and chi fields. HDF5 is not used: each field is a
        raw little-endian FP64 array ``vel_/pres_/chi_<name>.raw`` ([z][y][x], velocity
        with its 3 components innermost) with an XDMF descriptor ``.xmf`` beside it.
        Returns the path prefix ``<path4serialization>/<name>``."""
        name = (append if append else "restart_") + f"{self.step:09d}"
        base = self.sd.path4serialization
        os.makedirs(base, exist_ok=True)
        fpath = os.path.join(base, name)
        uinf = self.obstacle_state()["uinf"] if self.obstacles else np.array(self.sd.uinf, dtype=np.float64)
        status = (f"time: {self.time:20.20e}\nstepid: {int(self.step)}\nuinfx: {uinf[0]:20.20e}\n"
                  f"uinfy: {uinf[1]:20.20e}\nuinfz: {uinf[2]:20.20e}\n")
        if self.obstacles:
            pos = (C.c_double * 3)()
            L.check(L.lib().cup_get_sphere_position(self._h, pos), self._h, "serialize")
            sph = self.obstacles[0]
            mot = self.obstacle_state()
            vel, ang, q = list(mot["transVel"]), list(mot["angVel"]), list(mot["quaternion"])
            # absPos (the position in the lab frame, advanced by transVel alone;
            # exact for forced velocities, the latest velocity for free dofs)
            abspos = [p0 + self.time * vi for p0, vi in zip(sph.position, vel)]
            angle2d = 2 * np.arctan2(q[3], q[0])  # _2Dangle from the quaternion (Obstacle.cpp:348-350)
            lines = [f"{self.time:.16e}", "\t".join(f"{x:.16e}" for x in pos[:]),
                     "\t".join(f"{x:.16e}" for x in abspos), "\t".join(f"{x:.16e}" for x in q),
                     "\t".join(f"{x:.16e}" for x in vel), "\t".join(f"{x:.16e}" for x in ang), f"{angle2d:.16e}"]
            with open(fpath + "_0.txt", "w") as f:
                f.write("\n".join(lines) + "\n")
        with open(fpath + ".status", "w") as f:
            f.write(status)
        u, v, w = self.velocity()
        fields = {"vel_": (np.stack([u, v, w], axis=-1), "Vector"), "pres_": (self.pressure(), "Scalar"),
                  "chi_": (self.chi() if self.obstacles else np.zeros(self.shape), "Scalar")}
        for prefix, (arr, kind) in fields.items():
            stem = prefix + name
            np.ascontiguousarray(arr, dtype="<f8").tofile(os.path.join(base, stem + ".raw"))
            self._write_xmf(os.path.join(base, stem + ".xmf"), stem + ".raw", kind)
        with open(os.path.join(base, "restart.status"), "w") as f:
            f.write(status)
        return fpath

    def _write_xmf(self, path: str, raw: str, kind: str):
        nx, ny, nz = self.cells
        dims = f"{nz} {ny} {nx}" + (" 3" if kind == "Vector" else "")
        with open(path, "w") as f:
            f.write('<?xml version="1.0" ?>\n<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>\n<Xdmf Version="2.0">\n <Domain>\n'
                    '  <Grid GridType="Uniform">\n'
                    f'   <Time Value="{self.time:.16e}"/>\n'
                    f'   <Topology TopologyType="3DCORECTMesh" Dimensions="{nz + 1} {ny + 1} {nx + 1}"/>\n'
                    '   <Geometry GeometryType="ORIGIN_DXDYDZ">\n'
                    '    <DataItem Dimensions="3" NumberType="Double" Precision="8" Format="XML">0 0 0</DataItem>\n'
                    f'    <DataItem Dimensions="3" NumberType="Double" Precision="8" Format="XML">'
                    f'{self.h:.16e} {self.h:.16e} {self.h:.16e}</DataItem>\n'
                    '   </Geometry>\n'
                    f'   <Attribute Name="data" AttributeType="{kind}" Center="Cell">\n'
                    f'    <DataItem Dimensions="{dims}" NumberType="Float" Precision="8" Endian="Little" '
                    f'Format="Binary">{raw}</DataItem>\n'
                    '   </Attribute>\n  </Grid>\n </Domain>\n</Xdmf>\n')

    def deserialize(self) -> bool:
        """Simulation::_deserialize (source/Simulation.cpp:526-580): reads
        ``restart.status`` in path4serialization, then the velocity dump of that step
        and the obstacle's position (Obstacle::restart, source/obstacles/Obstacle.cpp:425-447;
        add the obstacle first, as the reference builds it from its arguments).
        Returns False (a new run) when there is no restart.status."""
        base = self.sd.path4serialization
        st = os.path.join(base, "restart.status")
        if not os.path.exists(st):
            return False
        vals = {}
        with open(st) as f:
            for line in f:
                k, _, val = line.partition(":")
                vals[k.strip()] = val.strip()
        try:
            time, step = float(vals["time"]), int(vals["stepid"])
            uinf = [float(vals["uinfx"]), float(vals["uinfy"]), float(vals["uinfz"])]
        except (KeyError, ValueError) as e:
            raise ValueError(f"Error reading restart file {st}: {e}") from None
        if step < 0 or time < 0:
            raise ValueError(f"Error reading restart file {st}")
        name = f"restart_{step:09d}"
        nx, ny, nz = self.cells
        vel = np.fromfile(os.path.join(base, "vel_" + name + ".raw"), dtype="<f8")
        if vel.size != 3 * nx * ny * nz:
            raise ValueError(f"restart velocity dump has {vel.size} values, the grid needs {3 * nx * ny * nz}")
        vel = vel.reshape(nz, ny, nx, 3)
        self.set_velocity(vel[..., 0], vel[..., 1], vel[..., 2])
        if self.obstacles:
            txt = os.path.join(base, name + "_0.txt")
            if os.path.exists(txt):
                with open(txt) as f:
                    rows = f.read().split("\n")
                pos = (C.c_double * 3)(*[float(x) for x in rows[1].split()[:3]])
                L.check(L.lib().cup_set_sphere_position(self._h, pos), self._h, "deserialize")
                q = [float(x) for x in rows[3].split()[:4]]
                vel = [float(x) for x in rows[4].split()[:3]]
                ang = [float(x) for x in rows[5].split()[:3]]
                self.set_sphere_motion(vel, ang, q)
        else:
            L.check(L.lib().cup_set_uinf(self._h, (C.c_double * 3)(*uinf)), self._h, "deserialize")
            self.sd.uinf = tuple(uinf)
        self.step, self.time = step, time
        L.check(L.lib().cup_set_clock(self._h, step, time), self._h, "deserialize")
        self._next_save_time = time + self.sd.saveTime
        return True

    def _maybe_serialize(self, dt: float):
        """The dump decision of Simulation::timestep (source/Simulation.cpp:595-598, 611-613)."""
        f, tsave = int(self.sd.saveFreq), float(self.sd.saveTime)
        nxt = getattr(self, "_next_save_time", tsave)
        dump_freq = f > 0 and (self.step + 1) % f == 0
        dump_time = tsave > 0 and (self.time + dt) > nxt
        if dump_time:
            self._next_save_time = nxt + tsave
        return dump_freq or dump_time

    def diagnostics(self) -> dict:
        out = (C.c_double * 3)()
        L.check(L.lib().cup_diagnostics(self._h, out), self._h, "diagnostics")
        return {"ke": out[0], "div_l2": out[1], "div_max": out[2]}

    def dc_history(self) -> list:
        """Relative residuals at each defect-correction check of the last solve."""
        out = (C.c_double * 16)()
        n = C.c_int()
        L.check(L.lib().cup_dc_history(self._h, out, 16, C.byref(n)), self._h, "dc_history")
        return list(out[:n.value])

    def profile(self, on: bool = True):
        L.check(L.lib().cup_profile_enable(self._h, int(on)), self._h, "profile")

    def profile_report(self, reset: bool = True) -> dict:
        import json
        buf = C.create_string_buffer(1 << 16)
        L.check(L.lib().cup_profile_report(self._h, buf, len(buf), int(reset)), self._h, "profile_report")
        return json.loads(buf.value.decode())

    def launch_count(self) -> int:
        n = C.c_longlong()
        L.check(L.lib().cup_launch_count(self._h, C.byref(n)), self._h, "launch_count")
        return n.value

    def debug_shift(self, f, g: int, dx: int, dy: int, dz: int) -> np.ndarray:
        a = _as_host_f64(f, self.shape)
        out = np.empty_like(a)
        L.check(L.lib().cup_debug_shift(self._h, _ptr(a), _ptr(out), g, dx, dy, dz, L.CUP_WHERE_HOST), self._h,
                "debug_shift")
        return out


def blocks_to_global(blocks: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    b = np.ascontiguousarray(blocks, dtype=np.float64).ravel()
    out = np.empty((nz, ny, nx), dtype=np.float64)
    L.check(L.lib().cup_blocks_to_global(_ptr(b), _ptr(out), nx, ny, nz), None, "blocks_to_global")
    return out


def global_to_blocks(g: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(g, dtype=np.float64)
    nz, ny, nx = a.shape
    out = np.empty(a.size, dtype=np.float64)
    L.check(L.lib().cup_global_to_blocks(_ptr(a), _ptr(out), nx, ny, nz), None, "global_to_blocks")
    return out
