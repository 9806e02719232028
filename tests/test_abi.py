"""CPU tests of the C ABI library: it loads without a GPU, exports every
symbol include/cup_b200.h declares, and its host-only helpers work. No
compute call is made here (there is no GPU on this machine)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO


def header_symbols():
    txt = open(os.path.join(REPO, "include", "cup_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(cup_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from cubismup_3d_b200 import _lib
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES), set(syms) ^ set(_lib.SIGNATURES)


def test_block_layout_round_trip():
    import cubismup_3d_b200 as cup
    nx, ny, nz = 48, 16, 32
    g = np.random.default_rng(0).standard_normal((nz, ny, nx))
    b = cup.global_to_blocks(g)
    # FluidBlock data[z][y][x] per 16^3 block, blocks ordered x fastest
    blocks = b.reshape(nz // 16, ny // 16, nx // 16, 16, 16, 16)
    assert np.array_equal(blocks[1, 0, 2], g[16:32, 0:16, 32:48])
    assert np.array_equal(cup.blocks_to_global(b, nx, ny, nz), g)


def test_layout_rejects_bad_sizes():
    import cubismup_3d_b200 as cup
    with pytest.raises(ValueError):
        cup.blocks_to_global(np.zeros(10), 10, 16, 16)


def test_null_handle_is_an_error_not_a_crash():
    from cubismup_3d_b200 import _lib
    L = _lib.lib()
    assert L.cup_sync(None) == _lib.CUP_ERR_ARG
    assert L.cup_destroy(None) == _lib.CUP_OK
    assert L.cup_create(None, None) == _lib.CUP_ERR_ARG
    assert L.cup_last_error(None) == b"null handle"
    cells = (C.c_int * 3)()
    assert L.cup_get_dims(None, cells, None) == _lib.CUP_ERR_ARG


def test_simulation_data_contract():
    import cubismup_3d_b200 as cup
    sd = cup.SimulationData(CFL=0.5, cells=(64, 32, 16))
    assert sd.bpd == (4, 2, 1)
    assert sd.DLM == 1.0 and sd.rampup == 100  # struct defaults (SimulationData.h:98,143)
    with pytest.raises(ValueError):
        sd.setCells(40, 32, 16)
    sd.BCx_flag = "wall"
    with pytest.raises(ValueError):
        sd.to_config()
    sd.BCx_flag = "periodic"
    cfg = sd.to_config()
    assert (cfg.bpdx, cfg.bpdy, cfg.bpdz) == (4, 2, 1)


def test_sphere_arguments_like_bindings():
    import cubismup_3d_b200 as cup
    s = cup.Sphere(radius=0.1, position=(0.5, 0.5, 0.5), enforcedVelocity=(1, 0, 0),
                   bForcedInSimFrame=(True, True, True), bFixFrameOfRef=(True, True, True))
    assert s.length == pytest.approx(0.2)
    assert cup.Sphere(length=0.4).radius == pytest.approx(0.2)
    with pytest.raises(ValueError, match="Cannot specify both"):
        cup.Sphere(radius=0.1, length=0.3)
    with pytest.raises(ValueError, match="Expected a"):
        cup.Sphere()
    st = s.to_struct()
    assert list(st.bForcedInSimFrame) == [1, 1, 1]


def test_rollout_checkpoint_interval():
    # the smallest checkpoint interval whose checkpoints plus one recomputed
    # segment fit the memory budget; 1 (keep every state) when all fit
    from cubismup_3d_b200.adjoint import checkpoint_interval
    assert checkpoint_interval(64, 25_000_000, 10 ** 12) == 1
    assert checkpoint_interval(64, 25_000_000, 500_000_000) == 4  # 16 checkpoints + 3 recomputed states
    assert checkpoint_interval(100, 50_000_000, 10 ** 9) == 8
    with pytest.raises(MemoryError):
        checkpoint_interval(100, 50_000_000, 10 ** 6)
