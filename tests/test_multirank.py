"""The multi-process plumbing of ``bench.py`` on CPU (world_size 2, gloo).

On GPUs each rank is an independent replica of the simulation (the ranks
exchange no data): the only collectives are the barrier around
the timed region and the max over ranks of the device time. These tests run
the same helpers over gloo on the host, and the reference arm under two
ranks: rank 0 alone runs the CPU baseline and prints the JSON line.
"""
import contextlib
import io
import json
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import argparse
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # max over ranks of a per-rank time, as the timed region reports it
        t = bench.max_over_ranks(torch, world, torch.device("cpu"), 1.5 + rank)
        dist.barrier()
        # the reference arm under torchrun: rank 0 runs and prints, the others return
        args = argparse.Namespace(cells=32, steps=1, warmup=3, scheme="upwind3_rk2", gpus=world,
                                  precision="fp32_dc")
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            bench.run_reference(args, rank)
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": t, "stdout": buf.getvalue()}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r0 = json.load(open(tmp_path / "rank0.json"))
    r1 = json.load(open(tmp_path / "rank1.json"))
    assert r0["max"] == r1["max"] == 2.5
    assert r1["stdout"] == ""
    lines = [l for l in r0["stdout"].splitlines() if l.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
