"""A fixed workload to run under a profiler (ncu): warm-up steps, then the
steps to capture, of one of the benchmark's forms.

    python -m cubismup_3d_b200.profile_case --case turbulence --precision fp64 --cells 256 256 128 --steps 2
    python -m cubismup_3d_b200.profile_case --case sphere --precision fp32_dc --steps 2
    python -m cubismup_3d_b200.profile_case --case adjoint --precision fp32_dc --cells 256 256 128 --steps 2
    python -m cubismup_3d_b200.profile_case --case forces --precision fp64 --steps 1

turbulence: decaying turbulence (E(k) ~ k^4 exp(-2 (k/4)^2), u_rms = 1, nu = 1e-3,
CFL = 0.1, upwind3 + RK2) in a periodic box of side 2 pi along the longest
axis; sphere: the benchmark's sphere (R = 0.1 at (0.5, 0.5, 0.5), U = (1, 0, 0)
in a fixed frame, Re = 300, implicit penalization 1e6) on 256x128x128 cells by
default, from rest; adjoint: `--steps` discrete-adjoint steps of the
turbulence case; forces: the sphere case followed by `--steps` surface-force
evaluations. Steps run launch by launch (no graph replay), so that a profiler
sees each kernel; the line printed at the end names the case.
"""
from __future__ import annotations

import argparse

import numpy as np


def main():
    import cubismup_3d_b200 as cup
    from cubismup_3d_b200 import initial_conditions as ic

    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=["turbulence", "sphere", "adjoint", "forces"], default="turbulence")
    ap.add_argument("--precision", choices=["fp64", "fp32_dc"], default="fp32_dc")
    ap.add_argument("--cells", type=int, nargs=3, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--steps", type=int, default=2)
    args = ap.parse_args()
    sphere = args.case in ("sphere", "forces")
    cells = tuple(args.cells) if args.cells else ((256, 128, 128) if sphere else (256, 256, 256))
    sd = cup.SimulationData(CFL=0.1, cells=cells)
    if sphere:
        sd.extent, sd.nu, sd.lambda_, sd.bImplicitPenalization = 2.0, 2 * 0.1 / 300, 1e6, True
    else:
        sd.extent, sd.nu, sd.lambda_ = 2 * np.pi, 1e-3, 1.0
    sd.rampup, sd.DLM, sd.scheme, sd.precision = 0, 0.0, "upwind3_rk2", args.precision
    sim = cup.Simulation(sd)
    sim.use_graphs(False)
    if sphere:
        sim.add_obstacle(cup.Sphere(radius=0.1, position=(0.5, 0.5, 0.5), enforcedVelocity=(1.0, 0.0, 0.0),
                                    bForcedInSimFrame=(True, True, True), bFixFrameOfRef=(True, True, True)))
        z = np.zeros(sim.shape)
        sim.set_velocity(z, z, z)
    else:
        sim.set_velocity(*ic.decaying_turbulence(cells, seed=1234))
    if args.case == "adjoint":
        import torch
        sim.bind_torch_stream()
        sim.run_steps(args.warmup)
        dt = sim.calcMaxTimestep()
        state = sim.velocity_raw()
        lam = torch.randn_like(state)
        for _ in range(args.steps):
            sim.adjoint_step(state, dt, lam)
        torch.cuda.synchronize()
    elif args.case == "forces":
        sim.run_steps(args.warmup)
        for _ in range(args.steps):
            sim.compute_forces()
    else:
        sim.run_steps(args.warmup)
        sim.run_steps(args.steps)
    sim.sync()
    print(f"profile case {args.case} {args.precision} {cells[0]}x{cells[1]}x{cells[2]}: "
          f"{args.warmup} warm-up + {args.steps} profiled", flush=True)
    sim.close()


if __name__ == "__main__":
    main()
