"""The periodic Poisson solve of a z-slab decomposed grid, one rank per GPU.

The reference splits the grid over MPI ranks and solves with FFTW-MPI slabs
and a transposed spectrum (source/poisson/PoissonSolverPeriodic.cpp:94-121).
Here rank r of G holds the planes z in [r nz/G, (r+1) nz/G) of the RHS (all x
and y). The solve p = H(f . H(b)) with the separable Hartley transform H is:

* the x and y passes on the slab (local: cup_poisson_pass on a handle of
  nx x ny x nz/G cells);
* an all-to-all that turns the slabs into y-pencils: rank r sends the y block
  s of its slab to rank s, which stacks the G blocks it receives along z;
* the z pass with the spectral divide on the pencil (local: a handle of
  nx x ny/G x nz cells whose spectral window is y in [s ny/G, (s+1) ny/G) of
  the global grid);
* the inverse all-to-all and the y and x passes on the slab.

Each rank sends and receives (G-1)/G of its slab twice per solve: over NCCL on
NVLink the exchange is one all-to-all per direction; the received blocks land
in the rank's own memory before any kernel reads them. The exchange is
pluggable: ``TorchExchange`` (torch.distributed: NCCL all_to_all, or paired
send/recv where the backend has no all-to-all) and ``LocalExchange`` (G ranks
emulated in one process, for tests). The transforms are pluggable too: the
CUDA passes of the library (``CudaPasses``) or any object with the same two
methods.

``SlabSimulation`` runs the whole FP64 step on such a slab, the reference's
Cartesian decomposition (source/SimulationData.cpp:211-230) restricted to z:
the rank's handle holds its slab plus HALO ghost planes on each side
(cup_config.z_halo), the stencil operators run on all of it (the ghost planes
absorb the periodic wrap of the kernels, so the interior outputs are exact
while the stencils reach at most HALO planes out), and ghost planes are
refreshed from the neighbouring ranks by a halo exchange of whole planes
(contiguous in the [z][y][x] layout) before they are read: the velocity after
every step, the pressure after the solve. The Poisson solve is ``solve`` above.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

from . import _lib as L


class TorchExchange:
    """All-to-all of equally shaped blocks over torch.distributed."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def __call__(self, send: Sequence) -> List:
        import torch
        recv = [torch.empty_like(t) for t in send]
        if self.dist.get_backend(self.group) == "nccl":
            self.dist.all_to_all(recv, list(send), group=self.group)
            return recv
        # backends without all_to_all: paired sends and receives
        reqs = []
        for s in range(self.world):
            if s == self.rank:
                recv[s].copy_(send[s])
                continue
            reqs.append(self.dist.isend(send[s].contiguous(), s, group=self.group))
            reqs.append(self.dist.irecv(recv[s], s, group=self.group))
        for r in reqs:
            r.wait()
        return recv


    def halo(self, send_down, send_up):
        """Ghost planes from the neighbours: ``send_down`` (this rank's first
        interior planes) goes to rank - 1, ``send_up`` (its last ones) to rank +
        1 (periodic); returns (from the rank above, from the rank below), i.e.
        the upper and the lower ghost planes. Messages between two ranks pair up
        in posting order, which also holds when both neighbours are the same rank."""
        import torch
        dist = self.dist
        up, down = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        from_up, from_down = torch.empty_like(send_down), torch.empty_like(send_up)
        if self.world == 1:
            from_up.copy_(send_down)
            from_down.copy_(send_up)
            return from_up, from_down
        ops = [dist.P2POp(dist.isend, send_down.contiguous(), down, self.group),
               dist.P2POp(dist.isend, send_up.contiguous(), up, self.group),
               dist.P2POp(dist.irecv, from_up, up, self.group),
               dist.P2POp(dist.irecv, from_down, down, self.group)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        return from_up, from_down

    def max(self, value: float) -> float:
        """Maximum of a scalar over the ranks."""
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64,
                         device="cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        return float(t.item())


class LocalExchange:
    """G ranks emulated in one process: ``exchange_all(sends)`` takes every
    rank's send list and returns every rank's receive list; ``halo_all`` does
    the same for the ghost-plane exchange."""

    @staticmethod
    def exchange_all(sends: Sequence[Sequence]) -> List[List]:
        G = len(sends)
        return [[sends[r][s] for r in range(G)] for s in range(G)]

    @staticmethod
    def halo_all(sends: Sequence) -> List:
        """sends[r] = (send_down, send_up) of rank r; returns, per rank, (from
        the rank above, from the rank below)."""
        G = len(sends)
        return [(sends[(r + 1) % G][0], sends[(r - 1) % G][1]) for r in range(G)]


class CudaPasses:
    """The library's FP64 passes on two handles of one rank: the z-slab
    (nx x ny x nz/G) and the y-pencil (nx x ny/G x nz) with its spectral
    window."""

    def __init__(self, cells, h, rank, world, device=0):
        from .simulation import Simulation, SimulationData
        nx, ny, nz = cells
        if nz % world or ny % world:
            raise ValueError("ny and nz must be divisible by the number of ranks")
        nzl, nyl = nz // world, ny // world
        if min(nzl, nyl) < 16:
            raise ValueError("slabs and pencils must be at least 16 cells thick")

        def handle(c):
            sd = SimulationData(CFL=0.1, cells=c)
            sd.extent = h * max(c)  # the global cell size
            sd.DLM, sd.lambda_, sd.rampup, sd.device = 0.0, 1.0, 0, device
            return Simulation(sd)

        self.slab = handle((nx, ny, nzl))
        self.pencil = handle((nx, nyl, nz))
        L.check(L.lib().cup_set_spectral_window(self.pencil._h, rank * nyl, ny), self.pencil._h, "spectral window")

    def _pass(self, sim, buf, p):
        sim.bind_torch_stream()
        L.check(L.lib().cup_poisson_pass(sim._h, C.c_void_p(buf.data_ptr()), p), sim._h, "poisson pass")

    def xy(self, buf):
        """x then y pass on the slab (the forward and the inverse are the same transform)."""
        self._pass(self.slab, buf, 0)
        self._pass(self.slab, buf, 1)

    def yx(self, buf):
        self._pass(self.slab, buf, 1)
        self._pass(self.slab, buf, 0)

    def z(self, buf):
        self._pass(self.pencil, buf, 2)

    def close(self):
        self.slab.close()
        self.pencil.close()


def to_pencil_blocks(slab, world: int):
    """The y blocks of a slab (nz/G, ny, nx) to send, block s to rank s."""
    nyl = slab.shape[1] // world
    return [slab[:, s * nyl:(s + 1) * nyl, :].contiguous() for s in range(world)]


def from_pencil_blocks(recv):
    """The pencil (nz, ny/G, nx) from the blocks received from ranks 0..G-1."""
    import torch
    return torch.cat(list(recv), dim=0).contiguous()


def to_slab_blocks(pencil, world: int):
    """The z blocks of a pencil to send back, block r to rank r."""
    nzl = pencil.shape[0] // world
    return [pencil[r * nzl:(r + 1) * nzl].contiguous() for r in range(world)]


def from_slab_blocks(recv):
    import torch
    return torch.cat(list(recv), dim=1).contiguous()


def solve(rhs_slab, passes, exchange, world: int):
    """p on this rank's slab from its slab of the h^3-premultiplied RHS."""
    buf = rhs_slab.clone().contiguous()
    passes.xy(buf)
    pencil = from_pencil_blocks(exchange(to_pencil_blocks(buf, world)))
    passes.z(pencil)
    buf = from_slab_blocks(exchange(to_slab_blocks(pencil, world)))
    passes.yx(buf)
    return buf


def solve_emulated(rhs_slabs: Sequence, passes: Sequence):
    """G ranks in one process (LocalExchange): every rank's slab of p."""
    G = len(rhs_slabs)
    bufs = [r.clone().contiguous() for r in rhs_slabs]
    for b, ps in zip(bufs, passes):
        ps.xy(b)
    recv = LocalExchange.exchange_all([to_pencil_blocks(b, G) for b in bufs])
    pencils = [from_pencil_blocks(rv) for rv in recv]
    for pc, ps in zip(pencils, passes):
        ps.z(pc)
    recv = LocalExchange.exchange_all([to_slab_blocks(pc, G) for pc in pencils])
    bufs = [from_slab_blocks(rv) for rv in recv]
    for b, ps in zip(bufs, passes):
        ps.yx(b)
    return bufs


class SlabSimulation:
    """One rank's z-slab (nz/G planes) of a periodic FP64 simulation split over
    G ranks along z, with HALO ghost planes on each side. ``sd`` describes the
    whole grid (cells, extent, nu, CFL, scheme, ...); ``device`` the rank's GPU.

    A step (``step`` with a TorchExchange, or ``step_emulated`` for G slabs in
    one process): AdvectionDiffusion and PressureRHS on the slab with its ghost
    planes (upwind3 + RK2 reaches 4 planes out, the RHS one more: the interior
    RHS is exact), the decomposed Poisson solve of the interior RHS, the
    pressure's ghost planes from the neighbours, the gradient correction, and
    the velocity's ghost planes from the neighbours for the next step and its
    CFL maximum (over the ranks: Simulation::calcMaxTimestep,
    source/Simulation.cpp:403-424). No obstacle."""

    HALO = 8  # a multiple of 8 keeps the slab's planes a multiple of 16; the stencils need 5

    def __init__(self, sd, rank: int, world: int, device=None):
        import dataclasses
        from .simulation import Simulation
        nx, ny, nz = sd.cells
        if nz % world or ny % world:
            raise ValueError("ny and nz must be divisible by the number of ranks")
        self.nzl = nz // world
        if self.nzl < 16 or self.nzl % 16:
            raise ValueError("each rank's slab must be a multiple of 16 planes")
        if sd.precision != "fp64":
            raise ValueError("the z-slab step is FP64")
        self.sd, self.rank, self.world = sd, rank, world
        self.device = sd.device if device is None else device
        self.h = sd.extent / max(sd.cells)
        H = self.HALO
        ext = (nx, ny, self.nzl + 2 * H)
        local = dataclasses.replace(sd, cells=ext, extent=self.h * max(ext), z_halo=H, device=self.device,
                                    freqDiagnostics=0, saveFreq=0, saveTime=0.0)
        self.sim = Simulation(local)
        self.passes = CudaPasses(sd.cells, self.h, rank, world, device=self.device)
        self.step_count, self.time = 0, 0.0

    # -- fields -------------------------------------------------------------------
    def _field(self, which: int):
        import torch
        from .simulation import _DeviceArray
        ptr = C.c_void_p()
        L.check(L.lib().cup_field_ptr(self.sim._h, which, C.byref(ptr)), self.sim._h, "field pointer")
        return torch.as_tensor(_DeviceArray(ptr.value, self.sim.shape, self.device), device=f"cuda:{self.device}")

    def _velocity(self):
        return [self._field(f) for f in (L.CUP_FIELD_U, L.CUP_FIELD_V, L.CUP_FIELD_W)]

    @property
    def interior(self):
        return slice(self.HALO, self.HALO + self.nzl)

    def set_velocity(self, u, v, w):
        """From the whole grid's velocity (host arrays of shape (nz, ny, nx)): this
        rank's slab and its ghost planes (the periodic neighbours' planes)."""
        import numpy as np
        nz = self.sd.cells[2]
        z = (np.arange(-self.HALO, self.nzl + self.HALO) + self.rank * self.nzl) % nz
        self.sim.set_velocity(*(np.ascontiguousarray(np.asarray(a)[z]) for a in (u, v, w)))

    def velocity(self):
        """This rank's slab of the velocity (host arrays, nz/G planes)."""
        return [a[self.interior] for a in self.sim.velocity()]

    # -- the step's phases ----------------------------------------------------------
    def _halo_sends(self, fields):
        H, n = self.HALO, self.nzl
        return [(f[H:2 * H].clone(), f[n:n + H].clone()) for f in fields]

    def _halo_recv(self, fields, recvs):
        H, n = self.HALO, self.nzl
        for f, (from_up, from_down) in zip(fields, recvs):
            f[n + H:].copy_(from_up)
            f[:H].copy_(from_down)

    def _advect_rhs(self, dt: float):
        self.sim.bind_torch_stream()
        L.check(L.lib().cup_advect_diffuse(self.sim._h, float(dt)), self.sim._h, "AdvectionDiffusion")
        L.check(L.lib().cup_pressure_rhs(self.sim._h, float(dt)), self.sim._h, "PressureRHS")
        return self._field(L.CUP_FIELD_RHS)[self.interior].contiguous()

    def _set_pressure(self, p):
        self._field(L.CUP_FIELD_P)[self.interior].copy_(p)

    def _grad(self, dt: float):
        self.sim.bind_torch_stream()
        L.check(L.lib().cup_grad_correct(self.sim._h, float(dt)), self.sim._h, "PressureProjection")
        self.step_count += 1
        self.time += dt

    def local_umax(self) -> float:
        """max |u + uinf| over the slab and its ghost planes (neighbours' cells)."""
        return self.sim.max_velocity()

    def dt_from_umax(self, umax: float) -> float:
        """Simulation::calcMaxTimestep (source/Simulation.cpp:403-424) on the
        maximum over the ranks."""
        import math
        sd = self.sd
        dt_dif = self.h * self.h / sd.nu if sd.nu > 0 else math.inf
        dt_adv = self.h / (umax + 1e-8)
        cfl = sd.CFL
        if self.step_count < sd.rampup:
            x = (self.step_count + 1.0) / sd.rampup
            cfl = math.exp(math.log(1e-3) * (1 - x) + math.log(sd.CFL) * x)
        return cfl * min(dt_dif, dt_adv)

    # -- one rank per process -------------------------------------------------------
    def calc_max_timestep(self, exchange) -> float:
        return self.dt_from_umax(exchange.max(self.local_umax()))

    def step(self, dt: float, exchange):
        rhs = self._advect_rhs(dt)
        p = solve(rhs, self.passes, exchange, self.world)
        self._set_pressure(p)
        pf = [self._field(L.CUP_FIELD_P)]
        self._halo_recv(pf, [exchange.halo(*snd) for snd in self._halo_sends(pf)])
        self._grad(dt)
        vel = self._velocity()
        self._halo_recv(vel, [exchange.halo(*snd) for snd in self._halo_sends(vel)])

    def close(self):
        self.sim.close()
        self.passes.close()


def calc_max_timestep_emulated(slabs: Sequence[SlabSimulation]) -> float:
    return slabs[0].dt_from_umax(max(s.local_umax() for s in slabs))


def _halo_emulated(slabs: Sequence[SlabSimulation], fields: Sequence[Sequence]):
    """Ghost planes of fields[r] (lists of the same fields on every slab r) from the neighbouring slabs."""
    G = len(slabs)
    sends = [s._halo_sends(f) for s, f in zip(slabs, fields)]
    for k in range(len(fields[0])):
        recvs = LocalExchange.halo_all([sends[r][k] for r in range(G)])
        for r in range(G):
            slabs[r]._halo_recv([fields[r][k]], [recvs[r]])


def step_emulated(slabs: Sequence[SlabSimulation], dt: float):
    """One step of G slabs held in one process (LocalExchange), phase by phase."""
    rhs = [s._advect_rhs(dt) for s in slabs]
    for s, p in zip(slabs, solve_emulated(rhs, [s.passes for s in slabs])):
        s._set_pressure(p)
    _halo_emulated(slabs, [[s._field(L.CUP_FIELD_P)] for s in slabs])
    for s in slabs:
        s._grad(dt)
    _halo_emulated(slabs, [s._velocity() for s in slabs])
