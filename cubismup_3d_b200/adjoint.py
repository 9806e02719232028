"""Differentiable rollouts of the time step (no counterpart in the reference).

``rollout(sim, u0, dts)`` advances a velocity field through ``len(dts)`` steps
of ``Simulation.timestep`` with the given (fixed) time steps and is a
``torch.autograd.Function``: its backward runs the hand-written discrete
adjoint of the step (``cup_adjoint_step``: transpose of the upwind/central
advection and of the diffusion, the symmetric pressure projection, the Heun
RK2 transpose), so ``loss.backward()`` yields dloss/du0 on the device.

Memory: the forward keeps one velocity checkpoint every ``checkpoint_every``
steps; the backward walks the segments from the last to the first, restores
the segment's checkpoint, recomputes the segment's states forward and applies
the adjoint steps in reverse. Peak extra memory is (n/K + K) velocity fields
for n steps and checkpoint interval K, so long rollouts fit in HBM. By default
(``checkpoint_every=None``) K is the smallest interval whose checkpoints fit
in half of the device's free memory: K = 1 (every state kept, no
recomputation, the backward is the adjoint steps alone) whenever the rollout
fits, which on a 180 GB device covers the benchmark rollouts with room to
spare.

The forward and the recomputation advance the handle with ``Simulation._advance``
(the step and the clock only), so a rollout writes no restart dump and no
diagnostics.dat / forcingData.dat line. In FP32-DC form the recomputed states
match the forward ones to within the defect-correction tolerance, not bitwise:
restoring a checkpoint restarts the pressure warm start, so the recomputed
steps start their correction solves from another initial pressure.

The fixed-dt convention makes the rollout a smooth function of u0 except where
an upwind switch flips sign; the adjoint freezes the switch at the forward
state (the derivative from either side at a kink is the one-sided one).
With the sphere, ``obstacle_gradients`` gives the gradients of
J = <g, u_T> + sum over steps of w . F_n (F_n the penalization force of step n,
e.g. w = (1/n, 0, 0) for the time-averaged drag) with respect to the initial
velocity, the characteristic function chi and the sphere's target velocity
(``cup_adjoint_step_obstacle``), with the same checkpointing.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import torch

from . import _lib as L
from .simulation import Simulation


def checkpoint_interval(nsteps: int, state_bytes: int, budget_bytes: int) -> int:
    """The smallest checkpoint interval K whose peak extra memory
    (ceil(n / K) checkpoints plus K - 1 recomputed states) fits the budget."""
    if nsteps <= 0:
        return 1
    for K in range(1, nsteps + 1):
        need = (-(-nsteps // K) + (K - 1 if K > 1 else 0)) * state_bytes
        if need <= budget_bytes:
            return K
    raise MemoryError(f"a {nsteps}-step rollout of {state_bytes}-byte states does not fit {budget_bytes} bytes")


def _auto_interval(sim: Simulation, nsteps: int) -> int:
    free, _ = torch.cuda.mem_get_info(sim.sd.device)
    state = 3 * int(torch.tensor([], dtype=sim.storage_dtype).element_size()) * int(torch.Size(sim.shape).numel())
    return checkpoint_interval(nsteps, state, free // 2)


class Rollout(torch.autograd.Function):
    """u_T = step(dt_{n-1}) o ... o step(dt_0) (u0), u0 of shape (3, nz, ny, nx)."""

    @staticmethod
    def forward(ctx, u0: torch.Tensor, sim: Simulation, dts: Sequence[float], checkpoint_every: int):
        if sim.obstacles:
            raise ValueError("rollout: the discrete adjoint does not support obstacles")
        if sim.forcing:
            raise ValueError("rollout: spectral forcing has no discrete adjoint")
        K = _auto_interval(sim, len(dts)) if checkpoint_every is None else int(checkpoint_every)
        if K < 1:
            raise ValueError("checkpoint_every must be >= 1")
        dts = [float(d) for d in dts]
        sim.bind_torch_stream()
        clock = (sim.step, sim.time)
        sim.set_velocity_raw(u0.detach().to(sim.storage_dtype).contiguous())
        ckpts = []
        for s, dt in enumerate(dts):
            if s % K == 0:
                ckpts.append(sim.velocity_raw())
            sim._advance(dt)
        uT = sim.velocity_raw()
        ctx.sim, ctx.dts, ctx.K, ctx.ckpts, ctx.clock = sim, dts, K, ckpts, clock
        ctx.in_dtype = u0.dtype
        ctx.end_clock = (sim.step, sim.time)
        return uT.to(u0.dtype)

    @staticmethod
    def backward(ctx, grad_uT: torch.Tensor):
        sim, dts, K = ctx.sim, ctx.dts, ctx.K
        sim.bind_torch_stream()
        lam = grad_uT.detach().to(sim.storage_dtype).contiguous().clone()
        n = len(dts)
        for seg in reversed(range(len(ctx.ckpts))):
            s0, s1 = seg * K, min(n, seg * K + K)
            states = [ctx.ckpts[seg]]
            if s1 - s0 > 1:  # recompute the segment's states from its checkpoint
                _set_clock(sim, ctx.clock[0] + s0, ctx.clock[1] + sum(dts[:s0]))
                sim.set_velocity_raw(ctx.ckpts[seg])
                for s in range(s0, s1 - 1):
                    sim._advance(dts[s])
                    states.append(sim.velocity_raw())
            for s in reversed(range(s0, s1)):
                sim.adjoint_step(states[s - s0], dts[s], lam)
            ctx.ckpts[seg] = None  # its memory goes back as the backward proceeds
        _set_clock(sim, *ctx.end_clock)
        ctx.ckpts = None
        return lam.to(ctx.in_dtype), None, None, None


def obstacle_gradients(sim: Simulation, u0: torch.Tensor, dts: Sequence[float], w_force, grad_uT=None,
                       checkpoint_every: Optional[int] = None):
    """Gradients of J = <grad_uT, u_T> + sum_n w_force . F_n over ``len(dts)``
    steps of ``sim`` (which has the sphere) from ``u0`` (3, nz, ny, nx):
    returns (dJ/du0, dJ/dchi, dJ/dU) as CUDA tensors (storage dtype, FP64 of the
    grid's shape, FP64 of 3), plus the list of forces F_n of the forward."""
    if not sim.obstacles:
        raise ValueError("obstacle_gradients: the simulation has no obstacle")
    if sim.forcing:
        raise ValueError("obstacle_gradients: spectral forcing has no discrete adjoint")
    K = _auto_interval(sim, len(dts)) if checkpoint_every is None else int(checkpoint_every)
    if K < 1:
        raise ValueError("checkpoint_every must be >= 1")
    dts = [float(d) for d in dts]
    n = len(dts)
    sim.bind_torch_stream()
    clock = (sim.step, sim.time)
    sim.set_velocity_raw(u0.detach().to(sim.storage_dtype).contiguous())
    ckpts, forces = [], []
    for s, dt in enumerate(dts):
        if s % K == 0:
            ckpts.append(sim.velocity_raw())
        forces.append(sim._advance(dt, stats=True).force.copy())
    end_clock = (sim.step, sim.time)
    dev = u0.device
    lam = (torch.zeros((3,) + sim.shape, dtype=sim.storage_dtype, device=dev) if grad_uT is None
           else grad_uT.detach().to(sim.storage_dtype).contiguous().clone())
    g_chi = torch.zeros(sim.shape, dtype=torch.float64, device=dev)
    g_vel = torch.zeros(3, dtype=torch.float64, device=dev)
    for seg in reversed(range(len(ckpts))):
        s0, s1 = seg * K, min(n, seg * K + K)
        states = [ckpts[seg]]
        if s1 - s0 > 1:  # recompute the segment's states from its checkpoint
            _set_clock(sim, clock[0] + s0, clock[1] + sum(dts[:s0]))
            sim.set_velocity_raw(ckpts[seg])
            for s in range(s0, s1 - 1):
                sim._advance(dts[s])
                states.append(sim.velocity_raw())
        for s in reversed(range(s0, s1)):
            sim.adjoint_step_obstacle(states[s - s0], dts[s], lam, w_force, g_chi, g_vel)
        ckpts[seg] = None
    _set_clock(sim, *end_clock)
    return lam, g_chi, g_vel, forces


def _set_clock(sim: Simulation, step: int, time: float):
    L.check(L.lib().cup_set_clock(sim._h, C.c_int(int(step)), C.c_double(float(time))), sim._h, "set_clock")
    sim.step, sim.time = int(step), float(time)


def rollout(sim: Simulation, u0: torch.Tensor, dts: Sequence[float],
            checkpoint_every: Optional[int] = None) -> torch.Tensor:
    """Differentiable ``len(dts)``-step rollout of ``sim`` from ``u0`` (3, nz, ny, nx).

    ``checkpoint_every``: the checkpoint interval K (None: the smallest that
    fits half of the free device memory). The handle's velocity is left at the
    final state after the forward; after a backward with K > 1 it holds an
    intermediate state of the recomputation."""
    return Rollout.apply(u0, sim, list(dts), checkpoint_every)
