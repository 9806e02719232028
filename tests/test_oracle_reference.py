"""The oracle against the reference's own code (CPU): the reference's operator
sources compiled unmodified against oracle/ref_shim (oracle/_ref/libref.so,
built by ``make -C oracle ref`` where the reference tree is present) run on a
one-process grid of FluidBlocks beside the oracle on the same inputs.

AdvectionDiffusion (KernelAdvectDiffuse + the tmp -> u copy) and PressureRHS
(KernelPressureRHS) match bitwise. PressureProjection (PoissonSolverPeriodic:
_cub2fftw, r2c, _solve, c2r, _fftw2cub; KernelGradP) matches to rounding: its
FFT is the stand-in's direct DFT, not FFTW or the oracle's radix-2 FFT.
"""
import numpy as np
import pytest

from conftest import rel_l2

ref_mod = pytest.importorskip("oracle.reference")
pytestmark = pytest.mark.skipif(not ref_mod.available(), reason="reference tree and its build are absent")


@pytest.fixture(autouse=True)
def _in_tmp_dir(tmp_path, monkeypatch):
    """The reference's obstacle code writes its force and velocity logs
    (forceValues_0.dat, ...) into the working directory, from a buffer
    flushed here (otherwise at exit, wherever the process then is)."""
    monkeypatch.chdir(tmp_path)
    yield
    ref_mod.flush_logs()


def pair(oracle, cells, extent, nu, uinf):
    nx, ny, nz = cells
    orc = oracle.OracleSim(nx, ny, nz, extent, nu=nu, CFL=0.5, rampup=0, DLM=0.0, lambda_=1.0, uinf=uinf)
    ref = ref_mod.ReferenceSim(nx, ny, nz, extent, nu, uinf)
    return orc, ref


@pytest.mark.parametrize("cells,uinf", [((32, 32, 32), (0.3, -0.2, 0.1)), ((64, 32, 16), (0.0, 0.0, 0.0))])
def test_advection_and_rhs_bitwise_vs_reference(oracle, cells, uinf):
    nx, ny, nz = cells
    orc, ref = pair(oracle, cells, 2 * np.pi, 0.01, uinf)
    rng = np.random.default_rng(3)
    u, v, w = (0.5 * rng.standard_normal((nz, ny, nx)) for _ in range(3))
    orc.set_velocity(u, v, w)
    ref.set_velocity(u, v, w)
    dt = 1e-3
    orc.operator("AdvectionDiffusion", dt)
    ref.operator("AdvectionDiffusion", dt)
    for a, b in zip(orc.velocity(), ref.velocity()):
        assert np.array_equal(a, b)
    orc.operator("PressureRHS", dt)
    ref.operator("PressureRHS", dt)
    assert np.array_equal(orc.get("rhs"), ref.rhs())


def test_projection_and_steps_vs_reference(oracle):
    from cubismup_3d_b200 import initial_conditions as ic
    cells = (32, 32, 32)
    orc, ref = pair(oracle, cells, 2 * np.pi, 0.01, (0.0, 0.0, 0.0))
    u, v, w = ic.taylor_green(cells, 2 * np.pi / 32)
    rng = np.random.default_rng(5)
    u, v, w = (a + 0.05 * rng.standard_normal(a.shape) for a in (u, v, w))
    orc.set_velocity(u, v, w)
    ref.set_velocity(u, v, w)
    for step in range(3):
        dt = orc.calc_max_timestep()
        for name in ("AdvectionDiffusion", "PressureRHS", "PressureProjection"):
            orc.operator(name, dt)
            ref.operator(name, dt)
        assert rel_l2(orc.get("p"), ref.get("p")) < 1e-13
        for a, b in zip(orc.velocity(), ref.velocity()):
            assert rel_l2(a, b) < 1e-14


@pytest.mark.parametrize("fix_frame", [(1, 1, 1), (0, 0, 0)])
def test_sphere_pipeline_vs_reference(oracle, fix_frame):
    # The whole pipeline with a forced sphere, in a frame fixed to it or moving
    # through the frame: the reference's own Sphere, ObstacleVector,
    # CreateObstacles (SDF, chi, centre of mass, surface points), UpdateObstacles,
    # Penalization and ComputeForces against the oracle's restatements.
    cells, L, nu = (64, 32, 32), 2.0, 2 * 0.25 / 300
    nx, ny, nz = cells
    orc = oracle.OracleSim(nx, ny, nz, L, nu=nu, CFL=0.1, rampup=0, DLM=0.0, lambda_=1e6, implicit_penalization=True,
                           scheme="ref", sphere={"radius": 0.25, "position": (0.5, 0.5, 0.5),
                                                 "velocity": (1.0, 0.0, 0.0), "forced": (1, 1, 1),
                                                 "fix_frame": fix_frame})
    ref = ref_mod.ReferenceSim(nx, ny, nz, L, nu, (0.0, 0.0, 0.0), 1e6, True)
    ref.add_sphere(0.25, (0.5, 0.5, 0.5), (1.0, 0.0, 0.0), (1, 1, 1), fix_frame)
    z = np.zeros(orc.shape)
    orc.set_velocity(z, z, z)
    ref.set_velocity(z, z, z)
    assert np.array_equal(orc.get("chi"), ref.get("chi"))
    for step in range(3):
        dt = orc.calc_max_timestep()
        orc.timestep(dt)
        ref.timestep(dt)
        ob, st = ref.obstacle(), orc.stats()
        assert np.array_equal(orc.get("chi"), ref.get("chi"))
        assert np.allclose(st["com"], ob["com"], rtol=0, atol=1e-15)
        assert np.allclose(st["uinf"], ob["uinf"], rtol=0, atol=0)
        assert np.allclose(st["force"], ob["force"], rtol=1e-12, atol=1e-12 * abs(ob["force"][0]))
        for a, b in zip(orc.velocity(), ref.velocity()):
            assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(np.stack(ref.velocity()))
    f, rf = orc.compute_forces(), ob["forces"]
    assert np.abs(f[:26] - rf).max() <= 1e-13 * np.abs(rf[:3]).max()
    assert f[26] == pytest.approx(ob["mass"], rel=1e-14)


@pytest.mark.parametrize("forced,fix_frame", [((0, 1, 1), (0, 0, 0)), ((0, 0, 0), (0, 0, 0)), ((0, 0, 0), (1, 0, 0))])
def test_free_sphere_rigid_update_vs_reference(oracle, forced, fix_frame):
    # UpdateObstacles with free dofs: the momentum integrals of
    # KernelIntegrateFluidMomenta and the 6x6 balance of
    # Obstacle::computeVelocities (free translation, and rotation when no dof
    # is forced), position and orientation advanced by CreateObstacles, the
    # frame following a free dof (updateUinf), against the reference's code
    cells, L, nu = (64, 32, 32), 2.0, 1e-3
    nx, ny, nz = cells
    pos = (0.6, 0.5, 0.45)
    orc = oracle.OracleSim(nx, ny, nz, L, nu=nu, CFL=0.1, rampup=0, DLM=0.0, lambda_=1e6, implicit_penalization=True,
                           scheme="ref", sphere={"radius": 0.25, "position": pos, "velocity": (0.0, 0.0, 0.0),
                                                 "forced": forced, "fix_frame": fix_frame})
    ref = ref_mod.ReferenceSim(nx, ny, nz, L, nu, (0.0, 0.0, 0.0), 1e6, True)
    ref.add_sphere(0.25, pos, (0.0, 0.0, 0.0), forced, fix_frame)
    Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    u, v, w = 0.5 + 0.2 * np.sin(2 * np.pi * Y / ny), 0.3 * np.sin(2 * np.pi * X / nx), 0.1 * np.cos(2 * np.pi * Z / nz)
    orc.set_velocity(u, v, w)
    ref.set_velocity(u, v, w)
    for step in range(4):
        dt = orc.calc_max_timestep()
        orc.timestep(dt)
        ref.timestep(dt)
        st, ob = orc.stats(), ref.obstacle()
        scale = max(1.0, np.abs(ob["transVel"]).max())
        assert np.allclose(st["transVel"], ob["transVel"], rtol=0, atol=1e-13 * scale)
        assert np.allclose(st["angVel"], ob["angVel"], rtol=0, atol=1e-12)
        assert np.allclose(st["position"], ob["position"], rtol=0, atol=1e-15)
        assert np.allclose(st["uinf"], ob["uinf"], rtol=0, atol=1e-13 * scale)
        assert np.array_equal(orc.get("chi"), ref.get("chi"))
        for a, b in zip(orc.velocity(), ref.velocity()):
            assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(np.stack(ref.velocity()))
    if not any(forced):
        assert abs(st["angVel"][2]) > 0.1  # the shear spins a free sphere
