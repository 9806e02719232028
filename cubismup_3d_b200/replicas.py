"""Independent runs spread over the GPUs of one node, one process per GPU.

The gradient checks of the discrete adjoint need one pair of forward rollouts
per direction (the 16 velocity directions of the 128^3 Taylor-Green rollout,
the 8 chi directions of the sphere); the directions are independent, so each
rank of ``torch.distributed`` takes every ``world``-th of them on its own GPU
and one all-reduce gathers the results on every rank. Nothing else is
exchanged: each rank holds a full replica of the simulation.

With no process group (or a single rank) everything runs locally.
"""
from __future__ import annotations

from typing import Callable, List, Sequence

import numpy as np


def _dist():
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover - torch is a dependency
        return None
    return dist if dist.is_available() and dist.is_initialized() else None


def rank_and_world():
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def indices_of_rank(n: int, rank: int, world: int) -> List[int]:
    """The items of ``range(n)`` rank ``rank`` of ``world`` evaluates: every
    ``world``-th, starting at ``rank`` (balanced to within one item)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"invalid rank {rank} of {world}")
    return list(range(rank, n, world))


def gather_values(values: dict, n: int, device=None) -> np.ndarray:
    """Every rank's ``{index: value}`` assembled into one FP64 array of length n
    on every rank (a sum all-reduce of the values and of a coverage count;
    each index must be evaluated by exactly one rank)."""
    import torch
    d = _dist()
    buf = torch.zeros(2, n, dtype=torch.float64, device=device)
    for i, v in values.items():
        buf[0, i] = float(v)
        buf[1, i] = 1.0
    if d is not None:
        d.all_reduce(buf, op=d.ReduceOp.SUM)
    out = buf.cpu().numpy()
    if not np.all(out[1] == 1.0):
        raise RuntimeError(f"items evaluated {out[1].tolist()} times (each must be evaluated once)")
    return out[0].copy()


def distributed_map(evaluate: Callable[[int], float], n: int, device=None) -> np.ndarray:
    """``[evaluate(i) for i in range(n)]`` with the items spread over the ranks."""
    rank, world = rank_and_world()
    return gather_values({i: evaluate(i) for i in indices_of_rank(n, rank, world)}, n, device)


def central_differences(loss: Callable[[object], float], x0, directions: Sequence, eps: float,
                        device=None) -> np.ndarray:
    """Central differences (loss(x0 + eps d) - loss(x0 - eps d)) / (2 eps) of a
    scalar loss along each direction d of ``directions``, spread over the ranks
    (for directions built on demand, call distributed_map with a function
    that builds direction i)."""

    def one(i):
        d = directions[i]
        return (float(loss(x0 + eps * d)) - float(loss(x0 - eps * d))) / (2 * eps)

    return distributed_map(one, len(directions), device)
