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


class LocalExchange:
    """G ranks emulated in one process: ``exchange_all(sends)`` takes every
    rank's send list and returns every rank's receive list."""

    @staticmethod
    def exchange_all(sends: Sequence[Sequence]) -> List[List]:
        G = len(sends)
        return [[sends[r][s] for r in range(G)] for s in range(G)]


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
