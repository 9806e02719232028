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


def _replica_worker(rank, world, port, outdir):
    import datetime

    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    from cubismup_3d_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        evaluated = []

        def evaluate(i):
            evaluated.append(i)
            return float(i * i)

        vals = replicas.distributed_map(evaluate, 16)
        # central differences of a quadratic loss along 8 directions (the chi
        # directions of the sphere check) spread over the ranks
        rng = np.random.default_rng(7)
        A = rng.standard_normal((5, 5))
        x0 = rng.standard_normal(5)
        dirs = [rng.standard_normal(5) for _ in range(8)]
        fd = replicas.central_differences(lambda x: 0.5 * x @ A @ x, x0, dirs, 1e-3)
        with open(os.path.join(outdir, f"replica{rank}.json"), "w") as f:
            json.dump({"evaluated": evaluated, "vals": vals.tolist(), "fd": fd.tolist()}, f)
    finally:
        dist.destroy_process_group()


def test_replicas_split_and_gather_gloo(tmp_path):
    # the FD directions of the adjoint checks spread over two ranks: each rank
    # evaluates every other item, and every rank ends with all the values
    import numpy as np
    pytest.importorskip("torch")
    import torch.multiprocessing as mp
    mp.spawn(_replica_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r = [json.load(open(tmp_path / f"replica{k}.json")) for k in range(2)]
    assert r[0]["evaluated"] == list(range(0, 16, 2)) and r[1]["evaluated"] == list(range(1, 16, 2))
    assert r[0]["vals"] == r[1]["vals"] == [float(i * i) for i in range(16)]
    rng = np.random.default_rng(7)
    A = rng.standard_normal((5, 5))
    x0 = rng.standard_normal(5)
    dirs = [rng.standard_normal(5) for _ in range(8)]
    exact = [0.5 * float(d @ (A + A.T) @ x0) for d in dirs]
    assert r[0]["fd"] == r[1]["fd"]
    assert np.allclose(r[0]["fd"], exact, rtol=1e-9, atol=1e-9)


def test_replicas_single_process():
    sys.path.insert(0, REPO)
    from cubismup_3d_b200 import replicas
    assert replicas.indices_of_rank(5, 1, 2) == [1, 3]
    assert replicas.distributed_map(lambda i: 2.0 * i, 4).tolist() == [0.0, 2.0, 4.0, 6.0]
    with pytest.raises(ValueError):
        replicas.indices_of_rank(5, 2, 2)
