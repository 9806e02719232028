"""B200-native fractional-step solver for CubismUP_3D's uniform periodic grid.

The compute path is hand-written sm_100a CUDA in ``libcup_b200.so`` behind the
C ABI of ``include/cup_b200.h``; this package is the host-side mirror of the
reference's Python bindings (``cubismup3d.SimulationData``, ``Simulation``,
``Sphere``) and of its ``Operator`` pipeline.
"""
from .simulation import (  # noqa: F401
    AdvectionDiffusion,
    ComputeDissipation,
    CreateObstacles,
    ObstacleArguments,
    Operator,
    Penalization,
    PoissonSolverPeriodic,
    PressureProjection,
    PressureRHS,
    Simulation,
    SimulationData,
    SpectralForcing,
    Sphere,
    StepStats,
    UpdateObstacles,
    blocks_to_global,
    global_to_blocks,
)
from . import _lib  # noqa: F401

__all__ = [
    "AdvectionDiffusion", "ComputeDissipation", "CreateObstacles", "ObstacleArguments", "Operator", "Penalization",
    "PoissonSolverPeriodic", "PressureProjection", "PressureRHS", "Simulation", "SimulationData", "SpectralForcing",
    "Sphere", "StepStats", "UpdateObstacles", "blocks_to_global", "global_to_blocks",
]
