"""The allocation-free max-velocity entry point (cup_max_velocity_noalloc).

Some callers cannot call cudaMalloc (their device memory belongs to another
allocator or to a budget fixed up front, or their running loop must never
allocate); this entry point serves them with a fixed scratch array inside the
library. The test calls it through the C ABI on caller-owned device arrays and
checks it against the handle-based cup_max_velocity on two calls in a row, the
second on a smaller field so that stale partials of the first call would show.
This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def handle_max(cells, u, v, w, uinf):
    import cubismup_3d_b200 as cup
    sd = cup.SimulationData(CFL=0.1, cells=cells, uinf=uinf)
    with cup.Simulation(sd) as sim:
        sim.set_velocity(u, v, w)
        return sim.max_velocity()


def noalloc_max(u, v, w, uinf):
    import torch

    from cubismup_3d_b200 import _lib
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    tu, tv, tw = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (u, v, w))
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    ui = (C.c_double * 3)(*uinf)
    stream = torch.cuda.current_stream(dev)
    rc = _lib.lib().cup_max_velocity_noalloc(C.c_void_p(tu.data_ptr()), C.c_void_p(tv.data_ptr()),
                                            C.c_void_p(tw.data_ptr()), tu.numel(), ui, C.c_void_p(out.data_ptr()),
                                            C.c_void_p(stream.cuda_stream))
    assert rc == _lib.CUP_OK
    stream.synchronize()
    return float(out.item())


def test_noalloc_max_velocity_matches_handle_twice():
    rng = np.random.default_rng(17)
    # first call: 128 x 64 x 64 (8 partial chunks); second: 32^3 with smaller values
    cases = [((128, 64, 64), 1.0, (0.3, -0.2, 0.1)), ((32, 32, 32), 0.25, (0.0, 0.05, 0.0))]
    for cells, scale, uinf in cases:
        nx, ny, nz = cells
        u, v, w = (scale * rng.standard_normal((nz, ny, nx)) for _ in range(3))
        got = noalloc_max(u, v, w, uinf)
        ref = handle_max(cells, u, v, w, uinf)
        assert got == pytest.approx(ref, rel=1e-15, abs=0)


def test_noalloc_propagates_nan():
    # one NaN cell makes the result NaN (a finite maximum would hide it and
    # give a plausible CFL time step)
    rng = np.random.default_rng(3)
    nx, ny, nz = 64, 32, 32
    u, v, w = (rng.standard_normal((nz, ny, nx)) for _ in range(3))
    v[17, 5, 40] = np.nan
    assert np.isnan(noalloc_max(u, v, w, (0.0, 0.0, 0.0)))
    v[17, 5, 40] = 0.0
    assert noalloc_max(u, v, w, (0.0, 0.0, 0.0)) == pytest.approx(
        max(np.abs(a).max() for a in (u, v, w)), rel=1e-15, abs=0)


def test_noalloc_rejects_oversized_fields():
    from cubismup_3d_b200 import _lib
    ui = (C.c_double * 3)(0.0, 0.0, 0.0)
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = _lib.lib().cup_max_velocity_noalloc(dummy, dummy, dummy, (1 << 28) + 1, ui, dummy, None)
    assert rc == _lib.CUP_ERR_ARG
