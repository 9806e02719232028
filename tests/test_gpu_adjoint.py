"""Discrete adjoint of the step on the GPU, checked three ways:

* dot-product test against the oracle's FP64 tangent-linear model:
  <lam, TLM(du)> = <ADJ(lam), du> to rounding (FP64 handle);
* directional derivatives of a rollout loss against central finite
  differences of the GPU forward;
* the FP32 adjoint against the FP64 tangent-linear model.

The adjoint freezes the upwind switch at the forward state, the same
convention as the oracle's tangent-linear model, so the dot-product identity
is exact up to rounding.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def make_sim(cells, extent, precision="fp64", scheme="upwind3_rk2", nu=5e-3, uinf=(0.0, 0.0, 0.0), CFL=0.5):
    import cubismup_3d_b200 as cup
    sd = cup.SimulationData(CFL=CFL, cells=cells, uinf=uinf)
    sd.extent, sd.nu, sd.rampup, sd.precision, sd.scheme = extent, nu, 0, precision, scheme
    return cup.Simulation(sd)


def make_oracle(oracle, cells, extent, scheme="upwind3_rk2", nu=5e-3, uinf=(0.0, 0.0, 0.0), CFL=0.5):
    return oracle.OracleSim(*cells, extent, nu, CFL=CFL, lambda_=1e6, DLM=1.0, uinf=uinf, rampup=0, scheme=scheme)


def initial_state(cells, h, seed, amplitude=0.05):
    from cubismup_3d_b200.initial_conditions import perturbed_taylor_green
    return perturbed_taylor_green(cells, h, seed, amplitude=amplitude, kmax=8)


def to_dev(fields, dtype):
    import torch
    return torch.from_numpy(np.stack(fields)).to(device="cuda", dtype=dtype).contiguous()


def dot(a, b):
    return float(np.sum(np.asarray(a, dtype=np.float64) * np.asarray(b, dtype=np.float64)))


@pytest.mark.parametrize("scheme,uinf", [("upwind3_rk2", (0.0, 0.0, 0.0)), ("upwind3_rk2", (0.3, -0.2, 0.1)),
                                         ("ref", (0.0, 0.0, 0.0))])
def test_adjoint_step_dot_product_vs_oracle_tlm(oracle, scheme, uinf):
    import torch
    cells = (32, 32, 32)
    ext = 2 * np.pi
    sim = make_sim(cells, ext, scheme=scheme, uinf=uinf)
    orc = make_oracle(oracle, cells, ext, scheme=scheme, uinf=uinf)
    u = initial_state(cells, sim.h, seed=1)
    rng = np.random.default_rng(5)
    du = [rng.standard_normal(sim.shape) for _ in range(3)]
    lam = [rng.standard_normal(sim.shape) for _ in range(3)]
    orc.set_velocity(*u)
    dt = orc.calc_max_timestep()
    tl = orc.tangent_run([dt], *du)
    state = to_dev(u, torch.float64)
    lam_d = to_dev(lam, torch.float64)
    sim.adjoint_step(state, dt, lam_d)
    adj = lam_d.cpu().numpy()
    lhs = dot(np.stack(lam), np.stack(tl))
    rhs = dot(adj, np.stack(du))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), np.linalg.norm(np.stack(lam)) * np.linalg.norm(np.stack(tl)))
    # the state argument is read only
    assert torch.equal(state, to_dev(u, torch.float64))


def test_adjoint_step_leaves_handle_state(oracle):
    import torch
    cells = (32, 32, 16)
    sim = make_sim(cells, 1.0)
    u = initial_state(cells, sim.h, seed=3)
    sim.set_velocity(*u)
    before = sim.velocity_raw().clone()
    lam = torch.randn((3,) + sim.shape, dtype=torch.float64, device="cuda")
    sim.adjoint_step(to_dev(u, torch.float64), 1e-3, lam)
    assert torch.equal(sim.velocity_raw(), before)


def test_adjoint_argument_checks():
    import torch
    import cubismup_3d_b200 as cup
    cells = (32, 32, 16)
    sim = make_sim(cells, 1.0)
    x = torch.zeros((3,) + sim.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="alias"):
        sim.adjoint_step(x, 1e-3, x)
    with pytest.raises(ValueError):
        sim.adjoint_step(x, 1e-3, torch.zeros((3,) + sim.shape, dtype=torch.float32, device="cuda"))
    with pytest.raises(ValueError, match="dt"):
        sim.adjoint_step(x, 0.0, x.clone())
    sim.add_obstacle(cup.Sphere(radius=0.1, position=(0.5, 0.5, 0.25), enforcedVelocity=(1, 0, 0),
                                bForcedInSimFrame=(True, True, True)))
    with pytest.raises(ValueError, match="obstacle"):
        sim.adjoint_step(x, 1e-3, x.clone())


@pytest.mark.parametrize("scheme", ["upwind3_rk2", "ref"])
def test_rollout_adjoint_vs_oracle_tlm(oracle, scheme):
    """7 steps, checkpoints every 3 (a partial last segment): the gradient of
    <w, u_T> against the oracle's FP64 tangent-linear rollout."""
    import torch
    from cubismup_3d_b200.adjoint import rollout
    cells = (32, 32, 32)
    ext = 2 * np.pi
    sim = make_sim(cells, ext, scheme=scheme)
    orc = make_oracle(oracle, cells, ext, scheme=scheme)
    u = initial_state(cells, sim.h, seed=2)
    orc.set_velocity(*u)
    dt = orc.calc_max_timestep()
    dts = [dt * (1 + 0.05 * i) for i in range(7)]
    rng = np.random.default_rng(9)
    du = [rng.standard_normal(sim.shape) for _ in range(3)]
    wgt = [rng.standard_normal(sim.shape) for _ in range(3)]
    tl = orc.tangent_run(dts, *du)
    uT_orc = np.stack(orc.velocity())
    u0 = to_dev(u, torch.float64).requires_grad_(True)
    uT = rollout(sim, u0, dts, checkpoint_every=3)
    assert rel_l2(uT.detach().cpu().numpy(), uT_orc) < 1e-10
    (uT * to_dev(wgt, torch.float64)).sum().backward()
    g = u0.grad.cpu().numpy()
    lhs = dot(np.stack(wgt), np.stack(tl))
    rhs = dot(g, np.stack(du))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs) + 1e-13 * np.linalg.norm(np.stack(wgt)) * np.linalg.norm(np.stack(tl))


@pytest.mark.parametrize("scheme,eps,tol", [("ref", 1e-6, 1e-8), ("upwind3_rk2", 1e-4, 1e-4)])
def test_rollout_gradient_vs_central_differences_fp64(scheme, eps, tol):
    """Central differences of the GPU forward. The central scheme is smooth, so
    the FD error is O(eps^2) and the bar is tight; with upwind3 every advecting
    velocity that changes sign inside [-eps, eps] along the path is a kink, and
    the FD error levels off near 1e-5 independent of eps (the gradient itself
    equals the tangent-linear value to rounding: see the dot-product tests)."""
    import torch
    from cubismup_3d_b200.adjoint import rollout
    from cubismup_3d_b200.initial_conditions import random_solenoidal
    cells = (32, 32, 32)
    ext = 2 * np.pi
    sim = make_sim(cells, ext, scheme=scheme)
    u = initial_state(cells, sim.h, seed=1)
    target = to_dev(initial_state(cells, sim.h, seed=2), torch.float64)
    sim.set_velocity(*u)
    dt = sim.calcMaxTimestep()
    dts = [dt] * 10
    u0 = to_dev(u, torch.float64)

    def loss(x):
        return 0.5 * ((rollout(sim, x, dts, checkpoint_every=4) - target) ** 2).sum()

    x = u0.clone().requires_grad_(True)
    loss(x).backward()
    grad = x.grad
    for seed in range(3):
        d = to_dev(random_solenoidal(cells, 100 + seed, lambda k: np.ones_like(k), kmax=8, amplitude=1.0),
                   torch.float64)
        with torch.no_grad():
            fd = (loss(u0 + eps * d) - loss(u0 - eps * d)).item() / (2 * eps)
        ad = float((grad * d).sum())
        assert abs(fd - ad) <= tol * abs(ad), (seed, fd, ad)


def test_fp32_adjoint_vs_fp64_tlm(oracle):
    import torch
    from cubismup_3d_b200.adjoint import rollout
    cells = (64, 64, 32)
    ext = 2 * np.pi
    sim = make_sim(cells, ext, precision="fp32_dc")
    orc = make_oracle(oracle, cells, ext)
    u = initial_state(cells, sim.h, seed=4)
    orc.set_velocity(*u)
    dt = orc.calc_max_timestep()
    dts = [dt] * 6
    rng = np.random.default_rng(21)
    du = [rng.standard_normal(sim.shape) for _ in range(3)]
    wgt = [rng.standard_normal(sim.shape) for _ in range(3)]
    tl = orc.tangent_run(dts, *du)
    u0 = to_dev(u, torch.float32).requires_grad_(True)
    uT = rollout(sim, u0, dts, checkpoint_every=4)
    (uT.double() * to_dev(wgt, torch.float64)).sum().backward()
    g = u0.grad.double().cpu().numpy()
    lhs = dot(np.stack(wgt), np.stack(tl))
    rhs = dot(g, np.stack(du))
    # FP32 storage and arithmetic: about 1e-6 relative per element
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs), (lhs, rhs)


def test_adjoint_rollout_taylor_green_128(oracle):
    """Perturbed Taylor-Green at 128^3 (perturbation amplitude 0.05, |k| <= 8,
    seed 1), nu = 5e-3, 64 steps at the CFL-0.5 dt of the initial field,
    checkpoints every 8; loss 0.5 ||u_T - u_target||^2 with u_target the
    seed-2 field. Gradients w.r.t. u0 from the FP32 and FP64 forward are held
    to 1e-4 of central FD (eps = 1e-4, FP64 forward) on 16 random solenoidal
    directions (seeds 100..115), and to the oracle's FP64 tangent-linear
    rollout on one of them."""
    import torch
    from cubismup_3d_b200.adjoint import rollout
    from cubismup_3d_b200.initial_conditions import random_solenoidal
    cells = (128, 128, 128)
    ext = 2 * np.pi
    nsteps, K, eps = 64, 8, 1e-4
    s64 = make_sim(cells, ext)
    s32 = make_sim(cells, ext, precision="fp32_dc")
    u = initial_state(cells, s64.h, seed=1)
    tgt_np = np.stack(initial_state(cells, s64.h, seed=2))
    target = torch.from_numpy(tgt_np).cuda()
    s64.set_velocity(*u)
    dt = s64.calcMaxTimestep()
    dts = [dt] * nsteps
    u0 = to_dev(u, torch.float64)

    def loss(sim, x):
        return 0.5 * ((rollout(sim, x, dts, checkpoint_every=K).double() - target) ** 2).sum()

    grads = {}
    for name, sim, dtype in (("fp64", s64, torch.float64), ("fp32", s32, torch.float32)):
        x = u0.to(dtype).clone().requires_grad_(True)
        loss(sim, x).backward()
        grads[name] = x.grad.double()
    # the 16 directions through the replica map (one process here: all local;
    # under torch.distributed each GPU takes every world-th direction)
    from cubismup_3d_b200 import replicas

    def direction(i):
        return to_dev(random_solenoidal(cells, 100 + i, lambda k: np.ones_like(k), kmax=8, amplitude=1.0),
                      torch.float64)

    def central(i):
        d = direction(i)
        with torch.no_grad():
            return (loss(s64, u0 + eps * d) - loss(s64, u0 - eps * d)).item() / (2 * eps)

    fds = replicas.distributed_map(central, 16)
    worst = {"fp64": 0.0, "fp32": 0.0}
    for i, fd in enumerate(fds):
        d = direction(i)
        for name, g in grads.items():
            worst[name] = max(worst[name], abs(float((g * d).sum()) - fd) / abs(fd))
    d0 = direction(0)
    assert worst["fp64"] <= 1e-4 and worst["fp32"] <= 1e-4, worst
    # FP64 tangent-linear rollout of the oracle along the first direction
    orc = make_oracle(oracle, cells, ext)
    orc.set_velocity(*u)
    tl = np.stack(orc.tangent_run(dts, *d0.cpu().numpy()))
    uT = np.stack(orc.velocity())
    tlm = float(((uT - tgt_np) * tl).sum())
    assert abs(float((grads["fp64"] * d0).sum()) - tlm) <= 1e-9 * abs(tlm)
    assert abs(float((grads["fp32"] * d0).sum()) - tlm) <= 1e-4 * abs(tlm)


# ---- obstacle: penalization, its force and the RHS obstacle terms ----------

# off the grid's symmetry planes: a cell whose central chi differences cancel by
# symmetry is not a surface cell, and any perturbation would make it one (the
# RHS surface set is piecewise constant in chi)
OBST_SPHERE = dict(radius=0.25, position=(0.52, 0.49, 0.505), enforcedVelocity=(1.0, 0.0, 0.0),
                   bForcedInSimFrame=(True, True, True), bFixFrameOfRef=(True, True, True))


def make_obstacle_sim(precision="fp64", scheme="ref"):
    import cubismup_3d_b200 as cup
    sd = cup.SimulationData(CFL=0.1, cells=(32, 16, 16))
    sd.extent, sd.nu, sd.rampup, sd.DLM, sd.lambda_ = 2.0, 2e-3, 0, 0.0, 1e6
    sd.bImplicitPenalization, sd.precision, sd.scheme = True, precision, scheme
    sim = cup.Simulation(sd)
    sim.add_obstacle(cup.Sphere(**OBST_SPHERE))
    return sim


def obstacle_case(sim, seed=5):
    import torch
    from cubismup_3d_b200.initial_conditions import random_solenoidal
    u = random_solenoidal(sim.shape[::-1], seed, lambda k: k ** 2 * np.exp(-(k / 2.0) ** 2), rms=0.3)
    u0 = to_dev(u, torch.float64)
    rng = np.random.default_rng(seed + 1)
    g = to_dev([rng.standard_normal(sim.shape) for _ in range(3)], torch.float64)
    return u0, g


def obstacle_loss(sim, u0, g, dts, w, chi=None, vel=None):
    import torch
    if chi is not None:
        sim.set_chi(chi)
    if vel is not None:
        sim.set_sphere_velocity(vel)
    sim.set_velocity_raw(u0.to(sim.storage_dtype).contiguous())
    J = 0.0
    for dt in dts:
        J += float(np.dot(w, sim.timestep(dt).force))
    uT = sim.velocity_raw().double()
    return J + float((uT * g).sum())


def test_obstacle_adjoint_vs_central_differences():
    """dJ/du0, dJ/dchi (8 random directions on the cells of the smoothed
    interface, 0 < chi < 1) and dJ/dU of J = <g, u_T> + time-averaged drag over
    4 steps, FP64, against central finite differences of the GPU forward."""
    import torch
    from cubismup_3d_b200.adjoint import obstacle_gradients
    sim = make_obstacle_sim()
    u0, g = obstacle_case(sim)
    dts = [0.01] * 4
    w = np.array([1.0 / len(dts), 0.0, 0.0])
    chi0 = sim.chi()
    vel0 = np.array(OBST_SPHERE["enforcedVelocity"])
    lam, g_chi, g_vel, forces = obstacle_gradients(sim, u0, dts, w, grad_uT=g, checkpoint_every=2)
    assert abs(forces[-1][0]) > 0
    g_u0 = lam.double().cpu().numpy()
    g_chi = g_chi.cpu().numpy()
    g_vel = g_vel.cpu().numpy()
    rng = np.random.default_rng(11)
    # initial velocity
    d = rng.standard_normal((3,) + sim.shape)
    eps = 1e-6  # the white-noise direction makes the rollout strongly nonlinear
    dd = torch.from_numpy(d).cuda()
    fd = (obstacle_loss(sim, u0 + eps * dd, g, dts, w, chi0, vel0) -
          obstacle_loss(sim, u0 - eps * dd, g, dts, w, chi0, vel0)) / (2 * eps)
    ad = float(np.sum(g_u0 * d))
    assert abs(fd - ad) <= 1e-6 * abs(ad) + 1e-9, ("u0", fd, ad)
    # characteristic function: directions on the interface cells (inside the
    # body, chi = 1 and b1 = 0: the surface set changes with the sign of a
    # perturbation there, a kink)
    body = (chi0 > 1e-3) & (chi0 < 1 - 1e-3)
    for k in range(8):
        dc = np.where(body, rng.standard_normal(sim.shape), 0.0)
        e = 1e-6
        fd = (obstacle_loss(sim, u0, g, dts, w, chi0 + e * dc, vel0) -
              obstacle_loss(sim, u0, g, dts, w, chi0 - e * dc, vel0)) / (2 * e)
        ad = float(np.sum(g_chi * dc))
        assert abs(fd - ad) <= 1e-5 * abs(ad) + 1e-9, ("chi", k, fd, ad)
    # target velocity (x)
    e = 1e-6
    fd = (obstacle_loss(sim, u0, g, dts, w, chi0, vel0 + [e, 0, 0]) -
          obstacle_loss(sim, u0, g, dts, w, chi0, vel0 - [e, 0, 0])) / (2 * e)
    assert abs(fd - g_vel[0]) <= 1e-5 * abs(g_vel[0]) + 1e-9, ("U", fd, g_vel[0])


def test_obstacle_adjoint_zero_cross_velocity_upwind3():
    """dJ/du0 (upwind3 + RK2, FP64, sphere in a fixed frame) from an initial
    velocity with only an x component: a_y = a_z = 0 in every cell of the first
    step, where a up3(a; f) has a kink in the advecting velocity. The adjoint
    takes the mean of the one-sided derivatives there, the value central
    differences see. (The x component varies along x, so the first step's RHS
    is not zero: at a zero RHS the obstacle correction of the RHS is
    positively homogeneous but not linear, and no gradient exists.)"""
    import torch
    from cubismup_3d_b200.adjoint import obstacle_gradients
    sim = make_obstacle_sim(scheme="upwind3_rk2")
    rng = np.random.default_rng(17)
    nz, ny, nx = sim.shape
    X, Y, Z = np.meshgrid(np.arange(nx) / nx, np.arange(ny) / ny, np.arange(nz) / nz, indexing="ij")
    # phases keep every factor (and the RHS, its x difference) away from zero on the grid
    gx = 0.3 * np.sin(2 * np.pi * X + 0.4) * np.cos(2 * np.pi * Y + 0.3) * (1 + 0.5 * np.sin(2 * np.pi * Z))
    u0 = torch.zeros((3,) + sim.shape, dtype=torch.float64, device="cuda")
    u0[0] = torch.from_numpy(np.ascontiguousarray(gx.transpose(2, 1, 0))).cuda()
    g = to_dev([rng.standard_normal(sim.shape) for _ in range(3)], torch.float64)
    dts = [0.01] * 4
    w = np.array([1.0 / len(dts), 0.0, 0.0])
    chi0 = sim.chi()
    vel0 = np.array(OBST_SPHERE["enforcedVelocity"])
    lam, _, _, _ = obstacle_gradients(sim, u0, dts, w, grad_uT=g, checkpoint_every=2)
    d = rng.standard_normal((3,) + sim.shape)
    dd = torch.from_numpy(d).cuda()
    eps = 1e-6
    fd = (obstacle_loss(sim, u0 + eps * dd, g, dts, w, chi0, vel0) -
          obstacle_loss(sim, u0 - eps * dd, g, dts, w, chi0, vel0)) / (2 * eps)
    ad = float(np.sum(lam.double().cpu().numpy() * d))
    assert abs(fd - ad) <= 1e-6 * abs(ad) + 1e-9, ("u0", fd, ad)


def test_obstacle_adjoint_fp32_tracks_fp64():
    """The FP32-storage obstacle adjoint against the FP64 one (same gradients to
    FP32 accuracy)."""
    from cubismup_3d_b200.adjoint import obstacle_gradients
    dts = [0.01] * 3
    w = np.array([1.0 / len(dts), 0.0, 0.0])
    out = {}
    for prec in ("fp64", "fp32_dc"):
        sim = make_obstacle_sim(prec)
        u0, g = obstacle_case(sim)
        lam, g_chi, g_vel, _ = obstacle_gradients(sim, u0, dts, w, grad_uT=g, checkpoint_every=2)
        out[prec] = (lam.double().cpu().numpy(), g_chi.cpu().numpy(), g_vel.cpu().numpy())
        sim.close()
    for a, b in zip(out["fp32_dc"], out["fp64"]):
        assert rel_l2(a, b) < 1e-3, rel_l2(a, b)


def test_obstacle_adjoint_argument_checks():
    import torch
    sim = make_obstacle_sim()
    z = torch.zeros((3,) + sim.shape, dtype=torch.float64, device="cuda")
    lam = torch.zeros_like(z)
    with pytest.raises(ValueError):
        sim.adjoint_step(z, 0.01, lam)  # the plain adjoint refuses a handle with an obstacle
    with pytest.raises(ValueError):
        sim.adjoint_step_obstacle(z, 0.01, lam, (1, 0, 0), torch.zeros(3, device="cuda"),
                                  torch.zeros(3, dtype=torch.float64, device="cuda"))


def test_adjoint_refuses_spectral_forcing():
    # the forcing has no transpose: the rollout and the C entry point refuse it
    import ctypes as C

    import torch

    import cubismup_3d_b200 as cup
    from cubismup_3d_b200 import _lib
    from cubismup_3d_b200.adjoint import rollout
    sd = cup.SimulationData(CFL=0.5, cells=(32, 32, 32))
    sd.extent, sd.nu, sd.rampup, sd.turbKinEn_target = 2 * np.pi, 5e-3, 0, 0.5
    sim = cup.Simulation(sd)
    u0 = torch.zeros((3,) + sim.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="forcing"):
        rollout(sim, u0, [1e-3])
    lam = torch.zeros_like(u0)
    rc = _lib.lib().cup_adjoint_step(sim._h, *[C.c_void_p(u0[i].data_ptr()) for i in range(3)], 1e-3,
                                     *[C.c_void_p(lam[i].data_ptr()) for i in range(3)])
    assert rc == _lib.CUP_ERR_STATE
    assert b"forcing" in _lib.lib().cup_last_error(sim._h)
    sim.close()


def test_rollout_backward_leaves_output_files(tmp_path, monkeypatch):
    # the rollout's forward and recomputation write no diagnostics line and no
    # restart dump: the run's files and its restart point stay as they were
    import torch

    from cubismup_3d_b200.adjoint import rollout
    monkeypatch.chdir(tmp_path)
    cells = (32, 32, 16)
    sim = make_sim(cells, 1.0)
    sim.sd.freqDiagnostics = 1
    sim.sd.saveFreq = 2
    sim.sd.path4serialization = str(tmp_path)
    u = initial_state(cells, sim.h, seed=3)
    sim.set_velocity(*u)
    for _ in range(2):
        sim.timestep(sim.calcMaxTimestep())
    files = {p.name: p.read_bytes() for p in tmp_path.iterdir() if p.is_file()}
    assert "diagnostics.dat" in files and "restart.status" in files
    u0 = to_dev(u, torch.float64).requires_grad_(True)
    uT = rollout(sim, u0, [2e-3] * 6, checkpoint_every=2)
    (0.5 * (uT ** 2).sum()).backward()
    assert u0.grad is not None and torch.isfinite(u0.grad).all()
    after = {p.name: p.read_bytes() for p in tmp_path.iterdir() if p.is_file()}
    assert after == files


def test_sphere_adjoint_256x128x128_100_steps():
    """The penalized-obstacle adjoint at full size: the sphere of radius 0.1 in
    the 256x128x128 box of length 2 (U = (1, 0, 0) in a fixed frame, Re = 300,
    implicit penalization lambda = 1e6) from rest, 100 steps; J = the
    time-averaged drag. dJ/dchi on 8 random directions over the interface
    cells and dJ/dU (the imposed velocity), from the FP64 and the FP32-DC
    forward (checkpoints chosen by the memory budget), against central
    differences of the FP64 forward. (From rest the first step's RHS is zero,
    where the obstacle correction of the RHS is positively homogeneous but not
    linear: J has no gradient with respect to u0 there. Perturbations of chi
    and U leave that RHS zero.)"""
    import torch

    import cubismup_3d_b200 as cup
    from cubismup_3d_b200.adjoint import obstacle_gradients

    def sphere_sim(precision):
        sd = cup.SimulationData(CFL=0.1, cells=(256, 128, 128))
        sd.extent, sd.nu, sd.rampup, sd.DLM, sd.lambda_ = 2.0, 2 * 0.1 / 300, 0, 0.0, 1e6
        sd.bImplicitPenalization, sd.scheme, sd.precision = True, "upwind3_rk2", precision
        sim = cup.Simulation(sd)
        sim.add_obstacle(cup.Sphere(radius=0.1, position=(0.5, 0.5, 0.5), enforcedVelocity=(1.0, 0.0, 0.0),
                                    bForcedInSimFrame=(True, True, True), bFixFrameOfRef=(True, True, True)))
        return sim

    s64, s32 = sphere_sim("fp64"), sphere_sim("fp32_dc")
    n = 100
    dts = [0.1 * s64.h / 1.0] * n  # the CFL step of the flow past the sphere at U = 1
    w = np.array([1.0 / n, 0.0, 0.0])
    u0 = torch.zeros((3,) + s64.shape, dtype=torch.float64, device="cuda")
    chi0 = s64.chi()
    vel0 = np.array([1.0, 0.0, 0.0])

    def J(chi=None, vel=None):
        if chi is not None:
            s64.set_chi(chi)
        s64.set_sphere_velocity(vel if vel is not None else vel0)
        s64.set_velocity_raw(u0.contiguous())
        tot = 0.0
        for dt in dts:
            tot += float(np.dot(w, s64.timestep(dt).force))
        if chi is not None:
            s64.set_chi(chi0)
        return tot

    grads = {}
    for name, sim in (("fp64", s64), ("fp32", s32)):
        sim.set_chi(chi0)
        lam, g_chi, g_vel, forces = obstacle_gradients(sim, u0, dts, w)
        grads[name] = (lam.double().cpu().numpy(), g_chi.cpu().numpy(), g_vel.cpu().numpy())
        assert forces[-1][0] > 0  # drag on the sphere
    rng = np.random.default_rng(31)
    # chi directions on the interface cells (0 < chi < 1) whose six neighbours
    # are all surface cells of the RHS correction (non-zero central chi
    # differences), so that a perturbation leaves the set of surface cells,
    # which the linearisation freezes, as it is
    grad2 = sum((np.roll(chi0, -1, a) - np.roll(chi0, 1, a)) ** 2 for a in range(3))
    surf = grad2 > 0
    nb_surf = np.ones_like(surf)
    for a in range(3):
        nb_surf &= np.roll(surf, 1, a) & np.roll(surf, -1, a)
    interface = (chi0 > 1e-3) & (chi0 < 1 - 1e-3) & nb_surf
    assert interface.sum() > 1000
    err = {"fp64": {}, "fp32": {}}
    for k in range(8):
        dc = np.where(interface, rng.standard_normal(chi0.shape), 0.0)
        e = 1e-6
        fd = (J(chi=chi0 + e * dc) - J(chi=chi0 - e * dc)) / (2 * e)
        for name, (_, gc, _) in grads.items():
            err[name][f"chi{k}"] = abs(float(np.sum(gc * dc)) - fd) / abs(fd)
    e = 1e-6
    fd = (J(vel=vel0 + [e, 0, 0]) - J(vel=vel0 - [e, 0, 0])) / (2 * e)
    for name, (_, _, gv) in grads.items():
        err[name]["U"] = abs(gv[0] - fd) / abs(fd)
    assert max(err["fp64"].values()) <= 1e-4, err
    assert max(err["fp32"].values()) <= 1e-4, err
