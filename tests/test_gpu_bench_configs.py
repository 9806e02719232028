"""Parity at the benchmark configurations, through the C ABI against the FP64
oracle on the same seeded inputs:

* decaying turbulence at 256^3 (upwind3 + RK2, nu = 1e-3, CFL = 0.1):
  the FP64 form per field (u, v, w, p) per step for 5 steps at 1e-10 relative
  L2; the FP32 + defect-correction form after 200 steps of the oracle's dt
  sequence at 1e-6 relative L2 velocity error;
* the sphere at 256x128x128 (R = 0.1, U = (1, 0, 0) in a fixed frame, Re = 300,
  implicit penalization lambda = 1e6, from rest): the penalization drag every
  step and the divergence norms (cup_diagnostics) after 20 steps, at 1e-10
  (FP64) and 1e-5 (FP32-DC) relative.

These are the slow GPU tests (the 200-step oracle run is about 80 s of CPU work
on 16 cores).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

N = 256
NU = 1e-3


def c2_pair(oracle, precision):
    import cubismup_3d_b200 as cup
    from cubismup_3d_b200 import initial_conditions as ic
    sd = cup.SimulationData(CFL=0.1, cells=(N, N, N))
    sd.extent, sd.nu, sd.rampup, sd.DLM, sd.lambda_ = 2 * np.pi, NU, 0, 0.0, 1.0
    sd.scheme, sd.precision = "upwind3_rk2", precision
    sim = cup.Simulation(sd)
    orc = oracle.OracleSim(N, N, N, 2 * np.pi, nu=NU, CFL=0.1, rampup=0, DLM=0.0, lambda_=1.0, scheme="upwind3_rk2")
    u, v, w = ic.decaying_turbulence((N, N, N), seed=1234)
    sim.set_velocity(u, v, w)
    orc.set_velocity(u, v, w)
    return sim, orc


def test_decaying_turbulence_256_fp64_per_field_per_step(oracle):
    sim, orc = c2_pair(oracle, "fp64")
    for step in range(5):
        dt = orc.calc_max_timestep()
        assert sim.calcMaxTimestep() == pytest.approx(dt, rel=1e-12)
        sim.timestep(dt, stats=False)
        orc.timestep(dt)
        for name, a, b in zip("uvw", sim.velocity(), orc.velocity()):
            e = rel_l2(a, b)
            assert e < 1e-10, (step, name, e)
        e = rel_l2(sim.pressure(), orc.get("p"))
        assert e < 1e-10, (step, "p", e)
    d, od = sim.diagnostics(), orc.diagnostics()
    assert d["ke"] == pytest.approx(od["ke"], rel=1e-12)
    # the projection makes the central divergence vanish: both are at rounding
    # level against the velocity gradients (|u| ~ 1, h = 2 pi / 256)
    scale = max(np.abs(a).max() for a in orc.velocity()) * N / (2 * np.pi)
    assert d["div_max"] < 1e-10 * scale and od["div_max"] < 1e-10 * scale
    sim.close()


def test_decaying_turbulence_256_fp32_dc_200_steps(oracle):
    sim, orc = c2_pair(oracle, "fp32_dc")
    dts = orc.run(200)
    for dt in dts[:-1]:
        sim.timestep(float(dt), stats=False)
    st = sim.timestep(float(dts[-1]))
    assert st.n_unconverged == 0
    e = rel_l2(np.stack(sim.velocity()), np.stack(orc.velocity()))
    assert e < 1e-6, e
    sim.close()


SPHERE_CELLS = (256, 128, 128)
SPHERE_NU = 2 * 0.1 * 1.0 / 300


def c3_pair(oracle, precision):
    import cubismup_3d_b200 as cup
    sd = cup.SimulationData(CFL=0.1, cells=SPHERE_CELLS)
    sd.extent, sd.nu, sd.rampup, sd.DLM, sd.lambda_ = 2.0, SPHERE_NU, 0, 0.0, 1e6
    sd.bImplicitPenalization, sd.scheme, sd.precision = True, "upwind3_rk2", precision
    sim = cup.Simulation(sd)
    sim.add_obstacle(cup.Sphere(radius=0.1, position=(0.5, 0.5, 0.5), enforcedVelocity=(1.0, 0.0, 0.0),
                                bForcedInSimFrame=(True, True, True), bFixFrameOfRef=(True, True, True)))
    nx, ny, nz = SPHERE_CELLS
    orc = oracle.OracleSim(nx, ny, nz, 2.0, nu=SPHERE_NU, CFL=0.1, rampup=0, DLM=0.0, lambda_=1e6,
                           implicit_penalization=True, scheme="upwind3_rk2",
                           sphere={"radius": 0.1, "position": (0.5, 0.5, 0.5), "velocity": (1.0, 0.0, 0.0),
                                   "forced": (1, 1, 1), "fix_frame": (1, 1, 1)})
    z = np.zeros(orc.shape)
    sim.set_velocity(z, z, z)
    orc.set_velocity(z, z, z)
    return sim, orc


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32_dc", 1e-5)])
def test_sphere_256x128x128_drag_and_divergence(oracle, precision, tol):
    sim, orc = c3_pair(oracle, precision)
    for step in range(20):
        dt = orc.calc_max_timestep()
        st = sim.timestep(dt)
        orc.timestep(dt)
        drag = orc.stats()["force"][0]
        assert abs(st.force[0] - drag) <= tol * abs(drag), (step, st.force[0], drag)
    d, od = sim.diagnostics(), orc.diagnostics()
    for k in ("div_l2", "div_max", "ke"):
        assert abs(d[k] - od[k]) <= tol * abs(od[k]), (k, d[k], od[k])
    e = rel_l2(np.stack(sim.velocity()), np.stack(orc.velocity()))
    assert e < tol, e
    sim.close()
