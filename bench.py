#!/usr/bin/env python
"""Benchmark of the periodic fractional step (cell-steps/s) on B200.

Workload (default): decaying turbulence on [0, 2pi]^3 at 256^3, seeded random
solenoidal velocity with E(k) ~ k^4 exp(-2 (k/4)^2), u_rms = 1, nu = 1e-3,
CFL = 0.1, upwind3 + RK2 advection, periodic FFT pressure projection, in the
chosen form: FP32 storage and advection, FP32 FFT correction solves inside an
FP64 defect-correction loop (relative FP64 residual tolerance 1e-10, checked
every step). Data are synthetic (generated here, seed 1234 + rank); each
field is 67 MB (FP32) or 134 MB (FP64), so every pass streams well over L2
(126 MB) in total.

One JSON line on rank 0. `value` is device-timed (CUDA events on the
solver's stream, inputs resident); `e2e` runs the same steps through the
public API from pinned host buffers (velocity upload, per-step
calcMaxTimestep + timestep with its stats read back, velocity download).
Beside it: the FP64 plain step on the same workload and the relative L2
velocity error of the FP32 form against it after the same steps, the
defect-correction statistics, the cost of one discrete-adjoint step against
one forward step, the sphere configuration (256x128x128, both forms, drag and
divergence against the oracle) and, on one GPU, the FP64 CPU oracle run from
the same initial velocity for the same number of steps: its first steps time
the CPU baseline, its final velocity is the reference of `rel_l2_vs_oracle`.
`--impl reference` times the CPU oracle (the FP64 restatement of the
reference's algorithm) on all host cores instead.
Multi-GPU: one process per GPU, each an independent replica (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

# Algorithmic bytes per cell per launch (compulsory reads + writes, halo
# re-reads not counted) of each kernel, by storage width of the fields.
def kernel_bytes(name: str, fp32: bool) -> float:
    s = 4 if fp32 else 8  # velocity storage
    w = 4 if fp32 else 8  # FFT work array element
    table = {
        "advect_diffuse_ref": 6 * s,
        "upwind3_stage1": 6 * s,
        "upwind3_stage2": 9 * s,
        "pressure_rhs": 3 * s + 8,
        "rhs_dht_x": 3 * s + 8,          # FP64: u* in, RHS rows transformed in smem, x-transform out
        "dht_x": 2 * w,
        "dht_y": 2 * w,
        "dht_z_solve": 2 * w,
        "dht_z_solve_mixed": 4 + 8,         # FP32 forward in, FP64 (divided, inverse-transformed) out
        "dht_y_f64": 16,                    # FP64 inverse y pass of the correction solve
        "grad_p": 8 + 6 * s,
        # FP32 defect-correction passes
        "rhs_residual": 3 * s + 8 + 4,       # u*, p in; r (FP32) out (b = div u* in registers)
        "dc_residual": 8 + 3 * s + 4,        # p, u* in (b recomputed); r out
        "dht_x_update_p": 4 + 8 + 8,         # correction rows in, p read-modify-write
        "grad_p_check": 8 + 6 * s + 8 + 8,  # p, u* in (b recomputed), u out; previous p in, warm start out
    }
    return float(table.get(name, 0.0))


# DRAM traffic per cell of one launch: dram__bytes_read.sum + dram__bytes_write.sum
# of a stored ncu capture of the 256^3 FP32-DC step (ncu --section
# MemoryWorkloadAnalysis on the launches of one bench step, --clock-control
# none), divided by the cells; scaled by the cells of the run, since traffic
# grows with the cells streamed. A stored figure, not measured by this run.
MEASURED_DRAM_BYTES_PER_CELL_FP32DC = {
    "grad_p_check": 46.1, "upwind3_stage1": 21.7, "upwind3_stage2": 35.1, "rhs_residual": 23.5,
    "dht_x_update_p": 21.5, "dht_z_solve_mixed": 8.5, "dht_y_f64": 12.7, "dht_x": 4.7, "dht_y": 4.6,
}


def canonical_step_bytes(fp32: bool, scheme: str, n_solves: int = 1) -> float:
    """Algorithmic bytes per cell-step of the hot path's canonical pass structure
    (upwind3: 288 B FP64, 160 B FP32 with one correction solve, +64 B per
    further solve; ref scheme: 216 / 124)."""
    if scheme == "upwind3_rk2":
        base = 160.0 if fp32 else 288.0
    else:
        base = 124.0 if fp32 else 216.0
    return base + (64.0 * max(0, n_solves - 1) if fp32 else 0.0)


def measured_peak():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.window = []
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(1.5)  # nvidia-smi start-up: samples begin before the timed region
        except OSError:
            self.p = None

    def mark(self, t0: float, t1: float):
        """Wall-clock window of the timed region (samples inside it are preferred)."""
        self.window = [t0, t1]

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        import datetime
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        parsed = []
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                ts = None
            try:
                sm_v, mx_v = float(r[2]), float(r[3])
            except ValueError:
                continue
            act = [nm for nm, val in zip(names, r[6:10]) if val.lower() == "active"]
            parsed.append((ts, sm_v, mx_v, act))
        inside = [p for p in parsed if self.window and p[0] is not None and
                  self.window[0] - 0.06 <= p[0] <= self.window[1] + 0.06]
        use = inside if inside else parsed
        reasons = sorted({a for p in use for a in p[3]})
        return {"sm_mhz": statistics.median([p[1] for p in use]) if use else None,
                "sm_max_mhz": use[-1][2] if use else None, "reasons": reasons, "samples": len(use),
                "samples_in_window": len(inside)}


def make_ic(n: int, seed: int):
    from cubismup_3d_b200 import initial_conditions as ic
    return ic.decaying_turbulence((n, n, n), seed=seed)


def workload_config(args) -> dict:
    n = args.cells
    return {
        "workload": f"decaying turbulence {n}^3 periodic [0,2pi]^3, E(k)~k^4 exp(-2(k/4)^2), u_rms=1, "
                    f"nu=1e-3, CFL=0.1, {args.scheme}, {args.precision}",
        "cells": [n, n, n],
        "scheme": args.scheme,
        "precision": args.precision,
        "nu": 1e-3,
        "CFL": 0.1,
        "l2": "inputs larger than L2: every field is %d MB, a step streams >2 GB" % (n ** 3 * (4 if args.precision == "fp32_dc" else 8) // 2 ** 20),
        "parallelism": f"replicas x{args.gpus}",
    }


def oracle_run(n: int, scheme: str, u, v, w, nsteps: int, timed_steps: int):
    """The CPU oracle (FP64 restatement of the reference path) on all host
    cores from (u, v, w): one warm-up step, `timed_steps` timed steps (the CPU
    baseline), then on to `nsteps` steps in all (its own CFL dt every step).
    Returns (cell-steps/s of the timed steps, their seconds, threads, the
    velocity after nsteps, its time)."""
    from oracle import oracle as O
    O.set_num_threads(os.cpu_count() or 1)
    L = 2 * np.pi
    sim = O.OracleSim(n, n, n, L, nu=1e-3, CFL=0.1, rampup=0, DLM=0.0, lambda_=1.0, scheme=scheme)
    sim.set_velocity(u, v, w)
    sim.run(1)
    timed = max(1, min(timed_steps, nsteps - 1)) if nsteps > 1 else timed_steps
    t0 = time.perf_counter()
    sim.run(timed)
    el = time.perf_counter() - t0
    done = 1 + timed
    if nsteps > done:
        sim.run(nsteps - done)
    vel = sim.velocity()
    t = sim.stats()["time"]
    return n ** 3 * timed / el, el, O.num_threads(), vel, t


def rel_l2_fields(a, b) -> float:
    num = sum(float(np.sum((x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(y ** 2)) for y in b)
    return (num / den) ** 0.5


def cpu_reference_rate(n: int, scheme: str, steps: int, warmup: int, u, v, w):
    """Times the CPU oracle (FP64 restatement of the reference path) on all host cores."""
    from oracle import oracle as O
    O.set_num_threads(os.cpu_count() or 1)
    L = 2 * np.pi
    sim = O.OracleSim(n, n, n, L, nu=1e-3, CFL=0.1, rampup=0, DLM=0.0, lambda_=1.0, scheme=scheme)
    sim.set_velocity(u, v, w)
    sim.run(warmup)
    t0 = time.perf_counter()
    sim.run(steps)
    el = time.perf_counter() - t0
    return n ** 3 * steps / el, el, O.num_threads()


def run_reference(args, rank: int):
    if rank != 0:
        return
    n = args.cells
    u, v, w = make_ic(n, 1234)
    rate, el, thr = cpu_reference_rate(n, "upwind3_rk2" if args.scheme == "upwind3_rk2" else "ref", args.steps,
                                       args.warmup, u, v, w)
    line = {
        "metric": "cell-steps/s", "value": rate, "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": workload_config(args),
        "cpu_baseline": {"value": rate, "unit": "cell-steps/s", "cores": thr, "kind": "port",
                         "sample": f"{args.steps} full {n}^3 FP64 steps after {args.warmup} warm-up steps "
                                   "(oracle: C++/OpenMP restatement of the reference's operators; the reference's "
                                   "own operator sources build here only against stand-ins for Cubism, MPI and "
                                   "FFTW-MPI (a direct-DFT Poisson solve), which pin parity but do not measure its "
                                   "speed)"},
        "e2e": {"value": rate, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def make_sim(cup, n: int, precision: str, scheme: str, device: int):
    sd = cup.SimulationData(CFL=0.1, cells=(n, n, n))
    sd.extent, sd.nu, sd.rampup, sd.DLM, sd.lambda_ = 2 * np.pi, 1e-3, 0, 0.0, 1.0
    sd.scheme, sd.precision, sd.device = scheme, precision, device
    return cup.Simulation(sd)


def timed_run(torch, sim, stream, steps: int, barrier):
    """K device-chained steps bracketed by CUDA events on the solver's stream."""
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    st = sim.run_steps(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    return ev0.elapsed_time(ev1), st


def max_over_ranks(torch, world: int, dev, x: float) -> float:
    if world == 1:
        return x
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def adjoint_cost(torch, sim, stream, reps: int = 10) -> dict:
    """One discrete-adjoint step (cup_adjoint_step: stage recompute, projection
    of the adjoint field, two transposed stages) against one forward step with
    the same fixed dt, both CUDA-event timed on the solver's stream."""
    torch.cuda.set_stream(stream)
    sim.bind_torch_stream()
    dt = sim.calcMaxTimestep()
    state = sim.velocity_raw()
    lam = torch.randn_like(state)
    for _ in range(2):
        sim.timestep(dt, stats=False)
        sim.adjoint_step(state, dt, lam)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(reps):
        sim.timestep(dt, stats=False)
    ev[1].record(stream)
    ev[2].record(stream)
    for _ in range(reps):
        sim.adjoint_step(state, dt, lam)
    ev[3].record(stream)
    torch.cuda.synchronize()
    fwd = ev[0].elapsed_time(ev[1]) / reps
    adj = ev[2].elapsed_time(ev[3]) / reps
    out = {"forward_ms_per_step": fwd, "adjoint_ms_per_step": adj, "adjoint_over_forward": adj / fwd,
           "note": "adjoint step = stage-1 recompute + adjoint projection + two transposed RK stages"}
    # whole differentiable rollouts (torch.autograd through adjoint.rollout):
    # forward and backward time per step, the checkpoint interval chosen by the
    # memory budget (every state kept: no recomputation) and K = 8 (one
    # forward recompute per step in the backward)
    from cubismup_3d_b200.adjoint import _auto_interval, rollout
    n = 16
    u0 = sim.velocity_raw()
    for label, K in (("auto", None), ("K8", 8)):
        for rep in range(2):  # the first pass allocates and captures
            x = u0.clone().requires_grad_(True)
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            torch.cuda.synchronize()
            e[0].record(stream)
            loss = (rollout(sim, x, [dt] * n, checkpoint_every=K).double() ** 2).sum()
            e[1].record(stream)
            loss.backward()
            e[2].record(stream)
            torch.cuda.synchronize()
        f_ms, b_ms = e[0].elapsed_time(e[1]) / n, e[1].elapsed_time(e[2]) / n
        out[f"rollout_{label}"] = {"steps": n, "checkpoint_every": K if K else _auto_interval(sim, n),
                                   "forward_ms_per_step": f_ms, "backward_ms_per_step": b_ms,
                                   "backward_over_forward": b_ms / f_ms,
                                   "backward_over_forward_step": b_ms / fwd}
    return out


SPHERE_CELLS = (256, 128, 128)


def sphere_leg(torch, cup, stream, args, local_rank: int, barrier) -> dict:
    """Sphere of radius 0.1 at (0.5, 0.5, 0.5) in a 256x128x128 periodic box of
    length 2, imposed velocity (1, 0, 0) in a frame fixed to it (uinf = -U),
    Re = 300, implicit penalization lambda = 1e6, from rest; upwind3 + RK2.
    Both forms through run_steps (dt chained on the device), CUDA-event timed
    after the same warm-up as the main run; the penalization drag and the
    divergence norms against the FP64 oracle after the same steps."""
    # the 500 steps of the configuration: the last sphere_steps timed, the
    # impulsive start from rest (whose pressure changes too fast for one
    # correction solve per step) in the untimed warm-up
    n_steps = max(1, min(args.sphere_steps, 500 - max(args.warmup, 3)))
    n_warm = 500 - n_steps
    out = {"workload": "sphere R=0.1 at (0.5,0.5,0.5), 256x128x128, extent 2, U=(1,0,0), fixed frame, Re=300, "
                       "lambda=1e6 implicit, from rest, upwind3_rk2, 500 steps", "steps": n_steps, "warmup": n_warm}
    res = {}
    for prec in ("fp32_dc", "fp64"):
        sd = cup.SimulationData(CFL=0.1, cells=SPHERE_CELLS)
        sd.extent, sd.nu, sd.rampup, sd.DLM, sd.lambda_ = 2.0, 2 * 0.1 * 1.0 / 300, 0, 0.0, 1e6
        sd.bImplicitPenalization, sd.precision, sd.scheme, sd.device = True, prec, "upwind3_rk2", local_rank
        s = cup.Simulation(sd)
        s.set_stream(stream.cuda_stream)
        s.add_obstacle(cup.Sphere(radius=0.1, position=(0.5, 0.5, 0.5), enforcedVelocity=(1.0, 0.0, 0.0),
                                  bForcedInSimFrame=(True, True, True), bFixFrameOfRef=(True, True, True)))
        z = np.zeros(s.shape)
        s.set_velocity(z, z, z)
        st0 = s.run_steps(n_warm)
        s.prepare_run(n_steps)
        ms, st = timed_run(torch, s, stream, n_steps, barrier)
        res[prec] = {"ms_per_step": ms / n_steps, "cell_steps_per_s": float(np.prod(SPHERE_CELLS)) * n_steps / (ms * 1e-3),
                     "drag": float(st.force[0]), "diagnostics": s.diagnostics(), "time": st.time}
        if prec == "fp32_dc":
            res[prec]["solves_per_step_timed"] = (st.n_solves_total - (st0.n_solves_total if st0 else 0)) / n_steps
            res[prec]["steps_missing_tol"] = st.n_unconverged
        res[prec]["velocity"] = s.velocity()
        s.close()
    out["fp32_dc"] = {k: v for k, v in res["fp32_dc"].items() if k != "velocity"}
    out["fp64"] = {k: v for k, v in res["fp64"].items() if k != "velocity"}
    out["speedup_fp32_dc_over_fp64"] = res["fp64"]["ms_per_step"] / res["fp32_dc"]["ms_per_step"]
    out["rel_l2_velocity_fp32_dc_vs_fp64"] = rel_l2_fields(res["fp32_dc"]["velocity"], res["fp64"]["velocity"])
    if not args.no_oracle_parity and int(os.environ.get("WORLD_SIZE", "1")) == 1:
        from oracle import oracle as O
        O.set_num_threads(os.cpu_count() or 1)
        nx, ny, nz = SPHERE_CELLS
        orc = O.OracleSim(nx, ny, nz, 2.0, nu=2 * 0.1 * 1.0 / 300, CFL=0.1, rampup=0, DLM=0.0, lambda_=1e6,
                          implicit_penalization=True, scheme="upwind3_rk2",
                          sphere={"radius": 0.1, "position": (0.5, 0.5, 0.5), "velocity": (1.0, 0.0, 0.0),
                                  "forced": (1, 1, 1), "fix_frame": (1, 1, 1)})
        z = np.zeros(orc.shape)
        orc.set_velocity(z, z, z)
        orc.run(n_warm + n_steps)
        ost, od = orc.stats(), orc.diagnostics()
        vo = orc.velocity()
        drag_o = float(ost["force"][0])
        out["oracle"] = {"drag": drag_o, "div_l2": od["div_l2"], "div_max": od["div_max"], "time": ost["time"]}
        for prec in ("fp32_dc", "fp64"):
            d = res[prec]["diagnostics"]
            out[prec]["vs_oracle"] = {
                "drag_rel": abs(res[prec]["drag"] - drag_o) / abs(drag_o),
                "div_l2_rel": abs(d["div_l2"] - od["div_l2"]) / od["div_l2"],
                "div_max_rel": abs(d["div_max"] - od["div_max"]) / od["div_max"],
                "rel_l2_velocity": rel_l2_fields(res[prec]["velocity"], vo)}
    return out


def run_ours(args, rank: int, world: int, local_rank: int):
    import ctypes as C

    import torch

    import cubismup_3d_b200 as cup
    from cubismup_3d_b200 import _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.cells
    fp32 = args.precision == "fp32_dc"
    sim = make_sim(cup, n, args.precision, args.scheme, local_rank)
    stream = torch.cuda.Stream(device=dev)
    sim.set_stream(stream.cuda_stream)
    u, v, w = make_ic(n, 1234 + rank)
    pinned = [torch.from_numpy(a).pin_memory() for a in (u, v, w)]
    sim.set_velocity(*[p.numpy() for p in pinned])

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # warm-up (also builds the per-kernel launch configuration caches); then the
    # 6-step CUDA graph that the timed run replays is captured and instantiated
    # (nothing runs), so that the one-off capture cost stays out of the timed region
    st_w = None
    for _ in range(args.warmup):
        st_w = sim.run_steps(1)
    graph_ready = sim.prepare_run(args.steps)
    sim.sync()

    # ---- device-timed region: K steps chained on the device ----
    launches0 = sim.launch_count()
    clocks = ClockSampler(local_rank)
    w0 = time.time()
    ms, st = timed_run(torch, sim, stream, args.steps, barrier)
    w1 = time.time()
    clocks.mark(w0, w1)
    clk = clocks.stop()
    launches = sim.launch_count() - launches0
    ms = max_over_ranks(torch, world, dev, ms)
    value = world * n ** 3 * args.steps / (ms * 1e-3)
    u_final = sim.velocity()
    r64 = None

    # ---- per-kernel profile (separate run, CUDA events per launch) ----
    sim.profile(True)
    sim.run_steps(max(2, min(args.steps, 5)))
    prof = sim.profile_report(reset=True)
    sim.profile(False)

    # ---- end-to-end through the public API with pinned host buffers ----
    out = [torch.empty_like(p).pin_memory() for p in pinned]
    sim_e2e_steps = args.steps  # the same run length as the device-timed steps
    # untimed: timestep() replays a one-step graph per phase of the field
    # rotation (6 phases); they are captured here, before the timed region
    sim.set_velocity(*[p.numpy() for p in pinned])
    for _ in range(7):
        sim.timestep(sim.calcMaxTimestep())
    sim.sync()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.set_velocity(*[p.numpy() for p in pinned])
    for _ in range(sim_e2e_steps):
        dt = sim.calcMaxTimestep()
        sim.timestep(dt)
    L.check(L.lib().cup_get_velocity(sim._h, *[C.c_void_p(o.data_ptr()) for o in out], L.CUP_WHERE_HOST), sim._h)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ems = max_over_ranks(torch, world, dev, e0.elapsed_time(e1))
    e2e = world * n ** 3 * sim_e2e_steps / (ems * 1e-3)
    field_bytes = 3 * n ** 3 * 8
    h2d = (field_bytes + sim_e2e_steps * 8) / sim_e2e_steps
    # per step one read of the device state (464 B) by timestep: its stats and the
    # next step's dt, which calcMaxTimestep then returns without another read
    d2h = (field_bytes + sim_e2e_steps * 464) / sim_e2e_steps

    # ---- discrete adjoint against forward (same handle, fixed dt) ----
    adj = adjoint_cost(torch, sim, stream) if not args.no_adjoint else None
    sim.close()

    # ---- FP64 plain step on the same workload: speed and the FP32 form's error ----
    fp64 = None
    if fp32 and not args.no_fp64_compare:
        s64 = make_sim(cup, n, "fp64", args.scheme, local_rank)
        s64.set_stream(stream.cuda_stream)
        s64.set_velocity(*[p.numpy() for p in pinned])
        for _ in range(args.warmup):
            s64.run_steps(1)
        s64.prepare_run(args.steps)
        ms64, st64 = timed_run(torch, s64, stream, args.steps, barrier)
        ms64 = max_over_ranks(torch, world, dev, ms64)
        v64 = world * n ** 3 * args.steps / (ms64 * 1e-3)
        r64 = s64.velocity()
        fp64 = {"value": v64, "ms_per_step": ms64 / args.steps, "speedup_fp32_dc_over_fp64": value / v64,
                "rel_l2_velocity_fp32_dc_vs_fp64": rel_l2_fields(u_final, r64),
                "after_steps": args.warmup + args.steps, "time_fp32_dc": st.time, "time_fp64": st64.time}
        s64.close()

    # ---- C3: forced sphere in a fixed frame, FP32-DC and FP64 ----
    sphere = sphere_leg(torch, cup, stream, args, local_rank, barrier) if not args.no_sphere else None

    if rank != 0:
        return

    peak, peak_kind = measured_peak()
    # roofline of the dominant kernel: algorithmic bytes / average launch time
    # (averaged over the launches that did the pass's work: the kernels of a
    # converged defect-correction loop's later solves exit at entry)
    kern = []
    for name, rec in prof.items():
        b = kernel_bytes(name, fp32)
        avg_ms = rec["work_ms"] / rec["work_count"]
        kern.append((rec["ms"], name, avg_ms, b * n ** 3 / (avg_ms * 1e-3) / 1e9 if b else None, rec["count"],
                     rec["work_count"]))
    kern.sort(reverse=True)
    top = next(k for k in kern if k[3] is not None)
    total_ms = sum(k[0] for k in kern)
    n_solves = st.n_solves if fp32 else 1
    cb = canonical_step_bytes(fp32, args.scheme, n_solves)
    traffic = None
    if fp32 and args.scheme == "upwind3_rk2" and top[1] in MEASURED_DRAM_BYTES_PER_CELL_FP32DC:
        traffic = MEASURED_DRAM_BYTES_PER_CELL_FP32DC[top[1]] * n ** 3
    roof = {"bound": "hbm", "kernel": top[1], "achieved": top[3], "peak": peak, "unit": "GB/s",
            "frac": top[3] / peak, "peak_kind": peak_kind, "traffic": traffic,
            "traffic_source": "ncu capture at 256^3 scaled by cells" if traffic else None,
            "algorithmic_bytes": kernel_bytes(top[1], fp32) * n ** 3,
            "step_bytes_per_cell": cb,
            "step_achieved": cb * value / world / 1e9,
            "step_frac": cb * value / world / 1e9 / peak}
    line = {
        "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if fp32 else "f64", "data": "synthetic",
        "config": workload_config(args),
        "roofline": roof,
        "kernels": {k[1]: {"share": k[0] / total_ms, "avg_ms": k[2], "launches": k[4], "work_launches": k[5],
                           "GBps": k[3]} for k in kern},
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": sim_e2e_steps,
                "note": "one FP64 velocity upload and download per run (3 x %d MB each way) and per step the "
                        "step's device state read back (its stats and the next dt); the transfers weigh less "
                        "in longer runs"
                        % (n ** 3 * 8 // 2 ** 20)},
        "graphs_captured_before_timing": graph_ready,
        "gpu_launches": launches,
        "clocks": clk,
        "final_state": {"time": st.time, "kinetic_energy": st.kinetic_energy, "umax": st.umax},
    }
    if fp32:
        line["defect_correction"] = {"tol": 1e-10, "n_solves_last_step": st.n_solves,
                                     "rel_residual_last_step": st.rel_residual,
                                     "steps_missing_tol": st.n_unconverged,
                                     "solves_per_step_timed":
                                         (st.n_solves_total - (st_w.n_solves_total if st_w else 0)) / args.steps}
    if fp64 is not None:
        line["fp64_plain"] = fp64
    if adj is not None:
        line["adjoint"] = adj
    if sphere is not None:
        line["sphere"] = sphere
    if not args.no_cpu_baseline and world == 1:
        # the FP64 oracle from the same initial velocity: its first steps time
        # the CPU baseline; after the run's warmup + steps steps it is the
        # reference of the GPU results' errors
        nsteps = args.warmup + args.steps if not args.no_oracle_parity else 1 + args.cpu_steps
        rate, el, thr, vel_o, t_o = oracle_run(n, args.scheme, u, v, w, nsteps, args.cpu_steps)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-steps/s", "cores": thr, "kind": "port",
                                "sample": f"{args.cpu_steps} full {n}^3 FP64 steps after 1 warm-up step, "
                                          f"{el:.1f} s of CPU work (oracle C++/OpenMP restatement)"}
        if not args.no_oracle_parity and u_final is not None:
            par = {"oracle_steps": nsteps, "oracle_time": t_o, "gpu_time": st.time,
                   "rel_l2_velocity_vs_oracle": rel_l2_fields(u_final, vel_o),
                   "bar": "<= 1e-6 relative L2 velocity (FP32-DC against the FP64 oracle)"}
            if fp64 is not None:
                par["rel_l2_velocity_fp64_vs_oracle"] = rel_l2_fields(r64, vel_o)
            line["rel_l2_vs_oracle"] = par["rel_l2_velocity_vs_oracle"]
            line["parity"] = par
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32_dc", choices=["fp64", "fp32_dc"])
    ap.add_argument("--scheme", default="upwind3_rk2", choices=["upwind3_rk2", "ref"])
    ap.add_argument("--cells", type=int, default=256)
    ap.add_argument("--cpu-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-compare", action="store_true", help="skip the FP64 plain run beside FP32_DC")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-step timing")
    ap.add_argument("--no-sphere", action="store_true", help="skip the sphere (256x128x128) leg")
    ap.add_argument("--sphere-steps", type=int, default=100, help="timed steps of the sphere leg (of its 500)")
    ap.add_argument("--no-oracle-parity", action="store_true",
                    help="run the CPU oracle only for the CPU baseline, not for the error of the GPU results")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
