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


class NumpyPasses:
    """The slab solver's passes in numpy (separable Hartley transforms, the
    reference's spectral factor and null modes), on CPU torch tensors."""

    def __init__(self, cells, h, rank, world):
        import numpy as np
        self.np = np
        nx, ny, nz = cells
        self.nx, self.ny, self.nz, self.h = nx, ny, nz, h
        self.y0 = rank * ny // world

    def _dht(self, a, axis):
        f = self.np.fft.fft(a, axis=axis)
        return f.real - f.imag

    def xy(self, buf):
        a = buf.numpy()
        a[...] = self._dht(self._dht(a, 2), 1)

    def yx(self, buf):
        a = buf.numpy()
        a[...] = self._dht(self._dht(a, 1), 2)

    def z(self, buf):
        np = self.np
        a = buf.numpy()
        nzl, nyl, nx = a.shape
        kz = np.arange(self.nz)[:, None, None]
        ky = (self.y0 + np.arange(nyl))[None, :, None]
        kx = np.arange(nx)[None, None, :]
        c = lambda k, n: np.cos(4 * np.pi * k / n)  # noqa: E731
        D = 2 * (c(kx, self.nx) + c(ky, self.ny) + c(kz, self.nz)) - 6
        nf = 4 / (self.nx * self.h * self.ny * self.nz)
        with np.errstate(divide="ignore"):
            f = np.where(D < -1e-12, nf / D, 0.0)
        a[...] = self._dht(f * self._dht(a, 0), 0)


def _slab_worker(rank, world, port, outdir):
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    from cubismup_3d_b200 import slab
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cells, h = (32, 32, 64), 0.1
        nx, ny, nz = cells
        rhs = np.random.default_rng(3).standard_normal((nz, ny, nx))
        nzl = nz // world
        mine = torch.from_numpy(rhs[rank * nzl:(rank + 1) * nzl].copy())
        p = slab.solve(mine, NumpyPasses(cells, h, rank, world), slab.TorchExchange(), world)
        np.save(os.path.join(outdir, f"slab{rank}.npy"), p.numpy())
    finally:
        dist.destroy_process_group()


def test_slab_poisson_solve_gloo(tmp_path):
    # The z-slab decomposed Poisson solve on two ranks (gloo): x/y passes on
    # the slabs, all-to-all to y-pencils, z pass with the spectral divide,
    # all-to-all back; the assembled pressure against the oracle's solve.
    import numpy as np
    pytest.importorskip("torch")
    import torch.multiprocessing as mp
    sys.path.insert(0, REPO)
    from oracle import oracle as O
    mp.spawn(_slab_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    p = np.concatenate([np.load(tmp_path / f"slab{r}.npy") for r in range(2)], axis=0)
    rhs = np.random.default_rng(3).standard_normal((64, 32, 32))
    ref = O.poisson_solve(rhs, 0.1)
    assert np.linalg.norm(p - ref) / np.linalg.norm(ref) < 1e-12


def test_slab_blocks_round_trip():
    # the block bookkeeping of the two all-to-alls, emulated for 4 ranks
    import numpy as np
    import torch
    sys.path.insert(0, REPO)
    from cubismup_3d_b200 import slab
    G, (nz, ny, nx) = 4, (64, 32, 16)
    full = torch.from_numpy(np.arange(nz * ny * nx, dtype=np.float64).reshape(nz, ny, nx))
    slabs = [full[r * nz // G:(r + 1) * nz // G] for r in range(G)]
    recv = slab.LocalExchange.exchange_all([slab.to_pencil_blocks(s, G) for s in slabs])
    pencils = [slab.from_pencil_blocks(rv) for rv in recv]
    for s, pc in enumerate(pencils):
        assert torch.equal(pc, full[:, s * ny // G:(s + 1) * ny // G])
    recv = slab.LocalExchange.exchange_all([slab.to_slab_blocks(pc, G) for pc in pencils])
    for r, rv in enumerate(recv):
        assert torch.equal(slab.from_slab_blocks(rv), slabs[r])


def _halo_worker(rank, world, port, outdir):
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    from cubismup_3d_b200 import slab
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ex = slab.TorchExchange()
        H, n = 2, 5  # ghost planes, interior planes per rank; plane value = its global z
        mine = torch.arange(rank * n, (rank + 1) * n, dtype=torch.float64).reshape(n, 1, 1).expand(n, 3, 4)
        from_up, from_down = ex.halo(mine[:H].clone(), mine[n - H:].clone())
        umax = ex.max(float(rank) + 0.5)
        np.savez(os.path.join(outdir, f"halo{rank}.npz"), up=from_up.numpy(), down=from_down.numpy(), umax=umax)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_halo_exchange_gloo(tmp_path, world):
    # ghost planes of a z-slab from the periodic neighbours (with two ranks both
    # neighbours are the same rank), and the maximum over the ranks
    import numpy as np
    pytest.importorskip("torch")
    import torch.multiprocessing as mp
    mp.spawn(_halo_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    H, n, nz = 2, 5, 5 * world
    for r in range(world):
        d = np.load(tmp_path / f"halo{r}.npz")
        up = [(r * n + n + k) % nz for k in range(H)]      # the first planes of the rank above
        down = [(r * n - H + k) % nz for k in range(H)]    # the last planes of the rank below
        assert np.array_equal(d["up"][:, 0, 0], up) and np.array_equal(d["down"][:, 0, 0], down)
        assert float(d["umax"]) == world - 0.5


def test_slab_halo_exchange_emulated():
    import torch
    sys.path.insert(0, REPO)
    from cubismup_3d_b200 import slab
    for G in (1, 2, 3):
        sends = [(torch.full((1,), 10.0 * r), torch.full((1,), 10.0 * r + 1)) for r in range(G)]
        recvs = slab.LocalExchange.halo_all(sends)
        for r, (from_up, from_down) in enumerate(recvs):
            assert float(from_up) == 10.0 * ((r + 1) % G)        # the send_down of the rank above
            assert float(from_down) == 10.0 * ((r - 1) % G) + 1  # the send_up of the rank below
