#!/usr/bin/env python
"""Benchmark of the periodic fractional step (cell-steps/s) on B200.

Workload (default): decaying turbulence on [0, 2pi]^3 at 256^3, seeded random
solenoidal velocity with E(k) ~ k^4 exp(-2 (k/4)^2), u_rms = 1, nu = 1e-3,
CFL = 0.1, upwind3 + RK2 advection, periodic FFT pressure projection. Data
are synthetic (generated here, seed 1234 + rank); each field is 134 MB (FP64)
or 67 MB (FP32), so every pass streams well over L2 (126 MB) in total.

One JSON line on rank 0. `value` is device-timed (CUDA events on the
solver's stream, inputs resident); `e2e` runs the same steps through the
public API from pinned host buffers (velocity upload, per-step
calcMaxTimestep + timestep with its stats read back, velocity download).
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
        "dht_x": 2 * w,
        "dht_y": 2 * w,
        "dht_z_solve": 2 * w,
        "grad_p": 8 + 6 * s,
    }
    return float(table.get(name, 0.0))


def step_bytes(fp32: bool, scheme: str) -> float:
    ad = kernel_bytes("upwind3_stage1", fp32) + kernel_bytes("upwind3_stage2", fp32) if scheme == "upwind3_rk2" \
        else kernel_bytes("advect_diffuse_ref", fp32)
    return ad + kernel_bytes("pressure_rhs", fp32) + 2 * kernel_bytes("dht_x", fp32) + \
        2 * kernel_bytes("dht_y", fp32) + kernel_bytes("dht_z_solve", fp32) + kernel_bytes("grad_p", fp32)


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
                                   "(oracle: C++/OpenMP restatement; the reference itself needs MPI, FFTW-MPI, HDF5, "
                                   "GSL and Cubism, absent on this image)"},
        "e2e": {"value": rate, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int):
    import ctypes as C

    import torch

    import cubismup_3d_b200 as cup
    from cubismup_3d_b200 import _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.cells
    fp32 = args.precision == "fp32_dc"
    sd = cup.SimulationData(CFL=0.1, cells=(n, n, n))
    sd.extent, sd.nu, sd.rampup, sd.DLM, sd.lambda_ = 2 * np.pi, 1e-3, 0, 0.0, 1.0
    sd.scheme, sd.precision, sd.device = args.scheme, args.precision, local_rank
    sim = cup.Simulation(sd)
    stream = torch.cuda.Stream(device=dev)
    sim.set_stream(stream.cuda_stream)
    u, v, w = make_ic(n, 1234 + rank)
    pinned = [torch.from_numpy(a).pin_memory() for a in (u, v, w)]
    sim.set_velocity(*[p.numpy() for p in pinned])

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # warm-up (also builds the per-kernel launch configuration caches)
    for _ in range(args.warmup):
        sim.run_steps(1)
    sim.sync()

    # ---- device-timed region: K steps chained on the device ----
    launches0 = sim.launch_count()
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    ev0.record(stream)
    st = sim.run_steps(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    barrier()
    clocks.mark(w0, w1)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = sim.launch_count() - launches0
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n ** 3 * args.steps / (ms * 1e-3)

    # ---- per-kernel profile (separate run, CUDA events per launch) ----
    sim.profile(True)
    sim.run_steps(max(2, min(args.steps, 5)))
    prof = sim.profile_report(reset=True)
    sim.profile(False)

    # ---- end-to-end through the public API with pinned host buffers ----
    out = [torch.empty_like(p).pin_memory() for p in pinned]
    sim_e2e_steps = min(args.steps, 50)
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
    ems = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ems], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ems = float(t.item())
    e2e = world * n ** 3 * sim_e2e_steps / (ems * 1e-3)
    field_bytes = 3 * n ** 3 * 8
    h2d = (field_bytes + sim_e2e_steps * 8) / sim_e2e_steps
    d2h = (field_bytes + sim_e2e_steps * (8 + 256)) / sim_e2e_steps

    if rank != 0:
        sim.close()
        return

    peak, peak_kind = measured_peak()
    # roofline of the dominant kernel: algorithmic bytes / average launch time
    kern = []
    for name, rec in prof.items():
        b = kernel_bytes(name, fp32)
        avg_ms = rec["ms"] / rec["count"]
        kern.append((rec["ms"], name, avg_ms, b * n ** 3 / (avg_ms * 1e-3) / 1e9 if b else None))
    kern.sort(reverse=True)
    top = next(k for k in kern if k[3] is not None)
    total_ms = sum(k[0] for k in kern)
    roof = {"bound": "hbm", "kernel": top[1], "achieved": top[3], "peak": peak, "unit": "GB/s",
            "frac": top[3] / peak, "peak_kind": peak_kind, "traffic": None,
            "step_achieved": step_bytes(fp32, args.scheme) * value / world / 1e9,
            "step_frac": step_bytes(fp32, args.scheme) * value / world / 1e9 / peak}
    line = {
        "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if fp32 else "f64", "data": "synthetic",
        "config": workload_config(args),
        "roofline": roof,
        "kernels": {k[1]: {"share": k[0] / total_ms, "avg_ms": k[2], "GBps": k[3]} for k in kern},
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
        "final_state": {"time": st.time, "kinetic_energy": st.kinetic_energy, "umax": st.umax},
    }
    sim.close()
    if not args.no_cpu_baseline and world == 1:
        rate, el, thr = cpu_reference_rate(n, args.scheme, args.cpu_steps, 1, u, v, w)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-steps/s", "cores": thr, "kind": "port",
                                "sample": f"{args.cpu_steps} full {n}^3 FP64 steps after 1 warm-up step, "
                                          f"{el:.1f} s of CPU work (oracle C++/OpenMP restatement)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_dc"])
    ap.add_argument("--scheme", default="upwind3_rk2", choices=["upwind3_rk2", "ref"])
    ap.add_argument("--cells", type=int, default=256)
    ap.add_argument("--cpu-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
