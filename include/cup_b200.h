/*
 * cup_b200.h — C ABI of the B200-native fractional-step solver for a uniform
 * periodic grid of 16^3-cell blocks (CubismUP_3D's hot path).
 *
 * The library owns all device memory of a simulation handle. Host pointers
 * passed in are borrowed for the duration of the call; device pointers
 * (CUP_WHERE_DEVICE) must stay valid until the call's work on the handle's
 * stream has finished. Calls on one handle are stream-ordered and not
 * re-entrant; different handles are independent. Every call returns a status
 * code; cup_last_error() gives a message for the last failing call on a handle.
 *
 * Field layout everywhere: a dense array of nz*ny*nx values, x fastest, i.e.
 * f[(z*ny + y)*nx + x] for the cell whose centre is ((x+.5)h, (y+.5)h, (z+.5)h).
 * (The reference stores the same cells block-wise as FluidBlock data[z][y][x],
 * source/Definitions.h:102-167; cup_blocks_to_global / cup_global_to_blocks
 * convert between the two.)
 */
#ifndef CUP_B200_H
#define CUP_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference aborts instead (source/SimulationData.cpp:180-226,
 * source/poisson/PoissonSolverPeriodic.cpp:94-103, source/operators/Operator.h:40-46). */
enum {
  CUP_OK = 0,
  CUP_ERR_ARG = 1,           /* invalid argument or unsupported configuration */
  CUP_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  CUP_ERR_NONFINITE = 3,     /* NaN/Inf detected in a reduction */
  CUP_ERR_NOT_CONVERGED = 4, /* defect correction hit max iterations */
  CUP_ERR_STATE = 5,         /* call not valid in the handle's current state */
  CUP_ERR_TIMEOUT = 6        /* a device-side wait ran past its time limit */
};

/* Storage / arithmetic form of a handle. */
enum {
  CUP_PREC_FP64 = 0,    /* FP64 storage and arithmetic throughout */
  CUP_PREC_FP32_DC = 1  /* FP32 storage/advection, FP32 FFT inside FP64 defect correction */
};

/* Advection scheme. */
enum {
  CUP_SCHEME_REF = 0,         /* central 2nd order + explicit Euler: KernelAdvectDiffuse,
                                 source/operators/AdvectionDiffusion.cpp:111-144 */
  CUP_SCHEME_UPWIND3_RK2 = 1  /* 3rd-order upwind-biased advection + central diffusion, Heun RK2 */
};

enum { CUP_WHERE_HOST = 0, CUP_WHERE_DEVICE = 1 };

/* Mirrors the hot-path subset of SimulationData (source/SimulationData.h:46-179).
 * Only uniform periodic grids: BC*_flag = periodic, bUseFourierBC = true. */
typedef struct cup_config {
  int bpdx, bpdy, bpdz;   /* blocks per dimension (cells = 16*bpd); each a power of two, 16..256 cells */
  double maxextent;       /* longest side; h = maxextent / max(cells)  (SimulationData.cpp:184-198) */
  double nu;              /* kinematic viscosity */
  double CFL;             /* Courant number (SimulationData.cpp:89) */
  double lambda;          /* penalization coefficient (SimulationData.cpp:87) */
  double DLM;             /* if > 0, lambda = DLM/dt each step (Simulation.cpp:418-419) */
  double uinf[3];         /* frame velocity (SimulationData.cpp:90-92) */
  int rampup;             /* CFL ramp-up steps (SimulationData.cpp:108) */
  int bImplicitPenalization; /* SimulationData.cpp:73 */
  int precision;          /* CUP_PREC_* */
  int scheme;             /* CUP_SCHEME_* */
  double dc_tol;          /* FP32_DC: relative FP64 residual tolerance (default 1e-10 if <= 0) */
  int dc_max_iter;        /* FP32_DC: max correction solves per step (default 2 if <= 0). A residual
                             check follows every solve; without an obstacle the check after the last
                             solve runs inside the gradient pass, so dc_max_iter = 1 is one solve and
                             one check per step, still verified against dc_tol */
  int dc_min_iter;        /* FP32_DC: solves always done per step (default 1 if <= 0) */
  int device;             /* CUDA device ordinal */
  int z_halo;             /* 0: a whole periodic grid. > 0 (4 or more, FP64): the handle holds one rank's
                             z-slab of a grid split over ranks along z, with z_halo ghost planes on each
                             side included in bpdz; nz = 16*bpdz then needs only be a multiple of 16 (32..512)
                             and the handle has no z Fourier transform: the stencil operators
                             (cup_advect_diffuse, cup_pressure_rhs, cup_grad_correct, cup_max_velocity,
                             cup_calc_max_timestep) run on it, with the ghost planes filled by the caller and
                             the Poisson solve done over the ranks (the z-slab decomposed solve); the entry
                             points that need the whole grid (steps and runs, Poisson solves, adjoint steps,
                             obstacles, diagnostics and spectral sums) return CUP_ERR_STATE */
} cup_config;

/* One sphere obstacle (source/obstacles/Sphere.cpp, ObstacleArguments in
 * source/obstacles/Obstacle.h:60-75). Forced translations move with
 * enforcedVelocity; free ones take the velocity of the momentum balance of
 * UpdateObstacles every step, and so does the rotation when no translation is
 * forced (any forced dof blocks rotation, source/obstacles/Obstacle.cpp:131-137). */
typedef struct cup_sphere {
  double radius;
  double position[3];
  double enforcedVelocity[3];
  int bForcedInSimFrame[3];
  int bFixFrameOfRef[3];
} cup_sphere;

typedef struct cup_solve_stats {
  int n_solves;            /* Poisson solves done (FP32_DC: correction solves) */
  double rel_residual;     /* final FP64 relative residual |b - L p| / |b| (FP32_DC), 0 for FP64 */
} cup_solve_stats;

typedef struct cup_step_stats {
  double dt, time;
  int step;
  double umax;             /* max |u + uinf| after the step (next calcMaxTimestep input) */
  double kinetic_energy;   /* sum h^3 |u|^2 / 2 after the step */
  double force[3], torque[3]; /* penalization force / torque on the sphere */
  int n_solves;
  double rel_residual;
  int n_unconverged;       /* steps since cup_create whose defect correction missed dc_tol */
  long long n_solves_total; /* FP32 correction solves since cup_create (FP32_DC) */
} cup_step_stats;

/* ---- lifetime (SimulationData ctor / Simulation ctor, source/Simulation.cpp:53-64) ---- */
int cup_create(const cup_config* cfg, struct cup_handle** out);
int cup_destroy(struct cup_handle* h);
const char* cup_last_error(const struct cup_handle* h);
/* Runs all subsequent work of the handle on this stream (cudaStream_t; NULL = the handle's own). */
int cup_set_stream(struct cup_handle* h, void* stream);
int cup_sync(struct cup_handle* h);
int cup_get_dims(const struct cup_handle* h, int cells[3], double* hgrid);

/* ---- fields ---- */
/* where = CUP_WHERE_HOST or CUP_WHERE_DEVICE; arrays are FP64 (double). */
int cup_set_velocity(struct cup_handle* h, const double* u, const double* v, const double* w, int where);
int cup_get_velocity(struct cup_handle* h, double* u, double* v, double* w, int where);
int cup_get_pressure(struct cup_handle* h, double* p, int where);
int cup_get_chi(struct cup_handle* h, double* chi, int where);
/* Pressure-RHS buffer (h^3 div u* / dt after PressureRHS), FP64 */
int cup_get_rhs(struct cup_handle* h, double* rhs, int where);

/* Device address of one of the handle's fields (no counterpart in the reference,
 * whose fields are the blocks' FluidElement members): CUP_FIELD_U/V/W (storage
 * type: FP64, or FP32 with CUP_PREC_FP32_DC), CUP_FIELD_P and CUP_FIELD_RHS
 * (FP64), each nz*ny*nx values in the field layout. The address holds until the
 * next call that advances the handle (a step or operator swaps the velocity
 * buffers); writes through it must be ordered with the handle's stream. Used to
 * exchange the ghost planes of a z-slab handle (cup_config.z_halo) in place. */
enum { CUP_FIELD_U = 0, CUP_FIELD_V = 1, CUP_FIELD_W = 2, CUP_FIELD_P = 3, CUP_FIELD_RHS = 4 };
int cup_field_ptr(struct cup_handle* h, int field, void** ptr);

/* Block-structured <-> global layout (Cubism FluidBlock data[z][y][x] per block,
 * blocks ordered x fastest): n = nx*ny*nz values. */
int cup_blocks_to_global(const double* blocks, double* global, int nx, int ny, int nz);
int cup_global_to_blocks(const double* global, double* blocks, int nx, int ny, int nz);

/* ---- obstacles ---- */
/* ObstacleVector::addObstacle (source/obstacles/ObstacleVector.h) for one sphere;
 * then CreateObstacles (source/operators/ObstaclesCreate.cpp:444-540) and
 * updateUinf (source/obstacles/ObstacleVector.h:60-76). At most one sphere. */
int cup_add_sphere(struct cup_handle* h, const cup_sphere* s);
/* CreateObstacles (source/operators/ObstaclesCreate.cpp:444-540) for a sphere
 * that moves in the frame (transVel + uinf != 0: a dof with a non-zero imposed
 * velocity and bFixFrameOfRef off): Obstacle::update
 * (source/obstacles/Obstacle.cpp:314-321) advances its position by
 * dt (transVel + uinf), then chi and the centre of mass are rebuilt. No-op for
 * a sphere at rest in the frame or without an obstacle. cup_step and cup_run
 * run it first in every step (cup_run then reads dt back once per step). */
int cup_create_obstacles(struct cup_handle* h, double dt);
/* Obstacle::restart's position (source/obstacles/Obstacle.cpp:425-447): moves
 * the sphere to `position` and rebuilds chi and the centre of mass there. */
int cup_set_sphere_position(struct cup_handle* h, const double position[3]);
/* The sphere's position (Obstacle::position; it follows Obstacle::update). */
int cup_get_sphere_position(struct cup_handle* h, double position[3]);
/* The frame velocity sim.uinf as restored by Simulation::_deserialize
 * (source/Simulation.cpp:526-580); only without an obstacle (updateUinf sets
 * it from the obstacle otherwise). */
int cup_set_uinf(struct cup_handle* h, const double uinf[3]);
/* UpdateObstacles (source/operators/ObstaclesUpdate.cpp:202-236) for a sphere
 * with free dofs, on the current velocity (before Penalization): the fluid
 * momentum integrals of KernelIntegrateFluidMomenta (:24-134) over chi > 0 and
 * the 6x6 momentum balance of Obstacle::computeVelocities
 * (source/obstacles/Obstacle.cpp:153-264), solved on the device; the free dofs
 * take the computed velocities. No-op for a fully forced sphere. cup_step and
 * cup_run run it between the projection and the penalization, and then read
 * the velocities back (one synchronisation per step for a free sphere).
 * Synchronises. */
int cup_update_obstacles(struct cup_handle* h, double dt);
/* The sphere's translational and angular velocity (Obstacle::transVel, angVel)
 * and orientation (Obstacle::quaternion, advanced by CreateObstacles). */
int cup_get_sphere_motion(struct cup_handle* h, double transVel[3], double angVel[3], double quaternion[4]);
/* Restores them (Obstacle::restart, source/obstacles/Obstacle.cpp:425-447);
 * for a frame fixed to a free dof, uinf follows (updateUinf). */
int cup_set_sphere_motion(struct cup_handle* h, const double transVel[3], const double angVel[3],
                          const double quaternion[4]);
/* Force / torque from the last Penalization (Penalization.cpp:101-123), centre of mass. */
int cup_get_obstacle_state(struct cup_handle* h, double force[3], double torque[3], double com[3],
                           double uinf[3]);

/* ---- operators (source/operators/*.cpp; names as Operator::getName()) ---- */
/* Sets the simulation clock (sim.step, sim.time) that calcMaxTimestep's CFL
 * ramp-up reads (source/Simulation.cpp:412-417) when the pipeline is driven
 * operator by operator rather than through cup_step / cup_run. */
int cup_set_clock(struct cup_handle* h, int step, double time);
/* findMaxU (source/operators/ProcessHelpers.h:74-99) */
int cup_max_velocity(struct cup_handle* h, double* umax);
/* Simulation::calcMaxTimestep (source/Simulation.cpp:403-424). Called right
 * after cup_step with stats (no other call between), it returns the dt that
 * step computed on the device from the same max |u| and step counter, which
 * the stats read-back already brought to the host: no device work and no
 * synchronisation. */
int cup_calc_max_timestep(struct cup_handle* h, double* dt);
/* AdvectionDiffusion::operator() (source/operators/AdvectionDiffusion.cpp:402-428) */
int cup_advect_diffuse(struct cup_handle* h, double dt);
/* PressureRHS::operator() (source/operators/PressureRHS.cpp:273-346) */
int cup_pressure_rhs(struct cup_handle* h, double dt);
/* PoissonSolverPeriodic::solve (source/poisson/PoissonSolverPeriodic.cpp:129-146) + _fftw2cub */
int cup_poisson_solve(struct cup_handle* h, cup_solve_stats* stats);
/* PoissonSolver's buffer contract (public data, stridex/y/z, data_size,
 * source/poisson/PoissonSolver.h:51-56; _offset/_dest, :72-101): *data = the
 * handle's FP64 device array that PressureRHS writes the h^3-premultiplied RHS
 * into and cup_poisson_solve reads; strides = {stridex, stridey, stridez} in
 * elements, so the cell (ix, iy, iz) of the block at index (bx, by, bz) is
 * data[16 (stridez bz + stridey by + stridex bx) + stridez iz + stridey iy +
 * stridex ix]; *data_size = its length. Valid for the handle's lifetime. A
 * caller may write its own RHS there (its kernels, cudaMemcpy, cup_set_rhs)
 * before cup_poisson_solve, as the reference's kernels write solver->data. In
 * the FP64 form the solve uses the array as its transform work space (as FFTW's
 * in-place buffer), so it does not hold the RHS afterwards; the solution is in
 * the pressure (cup_get_pressure: the solve includes _fftw2cub). */
int cup_poisson_buffer(struct cup_handle* h, double** data, size_t strides[3], size_t* data_size);
/* PoissonSolver::reset (source/poisson/PoissonSolver.cpp:132-135): zeroes the buffer. */
int cup_poisson_reset(struct cup_handle* h);
/* ---- the Poisson solve of a z-slab decomposed grid (PoissonSolverPeriodic
 * over MPI ranks, source/poisson/PoissonSolverPeriodic.cpp:94-121: FFTW-MPI
 * slabs with a transposed spectrum) ----
 * The solve p = H(f . H(b)) is separable: on a rank's z-slab (a handle of
 * nx x ny x nz/G cells) the x and y passes are local; after an all-to-all that
 * makes y-pencils (a handle of nx x ny/G x nz cells) the z pass with the
 * spectral divide is local too; a second all-to-all and the y and x passes
 * finish. cubismup_3d_b200/slab.py orchestrates it over torch.distributed. */
/* Makes the handle's z pass that of the pencil y in [y0, y0 + ny) of a grid
 * ny_global cells long in y (the global cos table, null modes and 1/N). */
int cup_set_spectral_window(struct cup_handle* h, int y0, int ny_global);
/* One FP64 pass of the Poisson solve, in place on the device array buf of the
 * handle's nx*ny*nz cells ([z][y][x]): pass 0 the Hartley transform of every
 * x row, 1 of every y column, 2 of every z column with the spectral divide of
 * PoissonSolverPeriodic::_solve between the forward and the inverse transform.
 * Stream-ordered on the handle's stream, no host synchronisation. */
int cup_poisson_pass(struct cup_handle* h, double* buf, int pass);
/* Writes the Poisson buffer (the mirror of cup_get_rhs); FP64, nx*ny*nz values. */
int cup_set_rhs(struct cup_handle* h, const double* rhs, int where);
/* KernelGradP (source/operators/PressureProjection.cpp:38-50) */
int cup_grad_correct(struct cup_handle* h, double dt);
/* PressureProjection::operator() (source/operators/PressureProjection.cpp:107-129) */
int cup_pressure_projection(struct cup_handle* h, double dt, cup_solve_stats* stats);
/* Penalization::operator() (source/operators/Penalization.cpp:129-156) */
int cup_penalize(struct cup_handle* h, double dt, double force_torque[6]);
/* Simulation::timestep (source/Simulation.cpp:593-623): the hot-path pipeline with
 * fused kernels. stats may be NULL (then no host synchronisation happens);
 * stats->dt is this step's dt. The step ends by computing the next step's CFL
 * dt on the device (read back with the stats for cup_calc_max_timestep). */
int cup_step(struct cup_handle* h, double dt, cup_step_stats* stats);
/* Simulation::run (source/Simulation.cpp:582-591) for nsteps: calcMaxTimestep + timestep,
 * with dt computed on the device (no host round trip per step). */
int cup_run(struct cup_handle* h, int nsteps, cup_step_stats* stats);
/* cup_run replays its steady-state steps from CUDA graphs of 6 steps and its
 * tail from one-step graphs (captured on first use; same kernels, same
 * results); off: every step is launched. */
int cup_set_graphs(struct cup_handle* h, int on);
/* Captures, without running anything, the CUDA graphs that cup_run(nsteps)
 * replays from the handle's current state (6-step graphs, then one-step graphs
 * for the run's tail), so that their capture, instantiation and upload are
 * paid here rather than in the run (no counterpart in the reference).
 * *captured (may be NULL) = the number of graphs the run will replay, all
 * cached now; 0 when the state cannot replay graphs yet (the FP32-DC warm
 * start is not ready, a moving obstacle, spectral forcing, profiling on,
 * graphs off). Nothing is launched on the stream. */
int cup_prepare_run(struct cup_handle* h, int nsteps, int* captured);

/* Discrete adjoint of one cup_step with the given dt (no counterpart in the
 * reference, which has no adjoint). un, vn, wn: the velocity at the start of the
 * step; lu, lv, lw: on entry dJ/du after the step, on return dJ/du before it. All
 * six are device arrays of nx*ny*nz elements in the handle's storage type (double
 * for CUP_PREC_FP64, float for CUP_PREC_FP32_DC), x fastest; the adjoint fields
 * must not alias the state. Upwind signs are frozen at the state; the projection
 * is applied as the exact (FP64 FFT) symmetric projector. The handle's own
 * velocity and pressure are untouched; its stage and RHS scratch are overwritten.
 * Handles with an obstacle return CUP_ERR_ARG; handles with spectral forcing on
 * return CUP_ERR_STATE (the forcing has no adjoint). Stream-ordered, no host sync. */
int cup_adjoint_step(struct cup_handle* h, const void* un, const void* vn, const void* wn, double dt, void* lu,
                     void* lv, void* lw);
/* Discrete adjoint of one cup_step of a handle with the sphere (no counterpart
 * in the reference): the same transposes as cup_adjoint_step plus those of the
 * Brinkman penalization (Penalization.cpp:40-98), of its force (:101-123) and of
 * the obstacle terms of the pressure RHS (PressureRHS.cpp:78-112, 215-256,
 * 322-343), for J = <g, u_T> + sum over steps of w_force . F_n (F_n the
 * penalization force of step n). un..lw as in cup_adjoint_step; w_force: 3 host
 * doubles; g_chi (device, nx*ny*nz doubles) += dJ/dchi on the obstacle's active
 * box (the derivative from the chi >= 0 side); g_vel (device, 3 doubles) +=
 * dJ/dU for the sphere's penalization target velocity U with uinf held fixed.
 * The step is recomputed from un (projection by the FP64 FFT solve); the surface
 * set and the sign of the RHS correction are frozen at it. CUP_ERR_STATE for a
 * moving sphere or with spectral forcing on. Stream-ordered. */
int cup_adjoint_step_obstacle(struct cup_handle* h, const void* un, const void* vn, const void* wn, double dt,
                              void* lu, void* lv, void* lw, const double w_force[3], double* g_chi, double* g_vel);
/* Replaces the obstacle's characteristic function (FP64, nx*ny*nz; only cells in
 * the obstacle's active box are read by the step). The centre of mass is kept. */
int cup_set_chi(struct cup_handle* h, const double* chi, int where);
/* Sets the sphere's penalization target velocity (transVel) without touching
 * uinf. */
int cup_set_sphere_velocity(struct cup_handle* h, const double vel[3]);
/* Device-to-device copies of the handle's velocity in its storage type (for
 * checkpoints): get copies out to u, v, w; set copies in. Stream-ordered. */
int cup_get_velocity_raw(struct cup_handle* h, void* u, void* v, void* w);
int cup_set_velocity_raw(struct cup_handle* h, const void* u, const void* v, const void* w);

/* Stand-alone Poisson solve: p = (wide-Laplacian)^+ rhs / h^3 on the handle's grid
 * (PoissonSolverPeriodic on an h^3-premultiplied RHS); rhs, p FP64. */
int cup_poisson_solve_field(struct cup_handle* h, const double* rhs, double* p, int where);

/* FP64 diagnostics of the current velocity: out[0] kinetic energy sum h^3|u|^2/2,
 * out[1] L2 norm (sum h^3 div^2)^(1/2) of the central divergence, out[2] max |div|
 * (ComputeDissipation.cpp:47-116 pattern, PoissonSolver.cpp:35-52 pattern). */
int cup_diagnostics(struct cup_handle* h, double out[3]);
/* ComputeForces (source/operators/FluidSolidForces.cpp:17-222) and
 * Obstacle::computeForces (source/obstacles/Obstacle.cpp:266-295) for the
 * sphere on the current fields: the surface points of CreateObstacles
 * (ObstaclesCreate.cpp:106-131) and the pressure and viscous stress on them.
 * out[27] = the 22 sums in ObstacleBlock::sumQoI order (surfForce[3],
 * presForce[3], viscForce[3], surfTorque[3], gamma[3], drag, thrust, Pout,
 * PoutBnd, defPower, defPowerBnd, pLocom), then Pthrust, Pdrag, EffPDef,
 * EffPDefBnd and the grid mass of chi. All zero without an obstacle. The reference runs it after
 * Penalization every step; cup_step / cup_run leave it out (they report the
 * penalization force), so call it after a step when the surface forces are
 * wanted. Synchronises the stream. */
int cup_compute_forces(struct cup_handle* h, double out[27]);
/* ComputeDissipation (source/operators/ComputeDissipation.cpp:38-177) on the
 * current fields: out[20] = circulation[3], linImpulse[3], linMomentum[3],
 * angImpulse[3], angMomentum[3], presPow, viscPow, helicity, kineticEn,
 * enstrophy (the reference's RDX order and diagnostics.dat columns), FP64. */
int cup_compute_dissipation(struct cup_handle* h, double out[20]);
/* SpectralAnalysis (source/spectralOperators/SpectralManipFFTW.cpp:110-193) of the
 * current velocity: stats = tke, eps, uprime, lambda, Re_lambda, l_integral,
 * tau_integral; spectrum (may be NULL) = E_msr, nbin = max(N)/2 - 1 shells
 * (HITstatistics, source/spectralOperators/SpectralManip.h:50-100). Computed on
 * the separable Hartley transform of the Poisson passes; the shell sums equal
 * the r2c ones. */
int cup_spectral_analysis(struct cup_handle* h, double stats[7], double* spectrum, int nbin);
/* SpectralForcing (source/spectralOperators/SpectralForcing.cpp:23-86) in every
 * cup_step / cup_run step after AdvectionDiffusion, to meet turbKinEn_target or
 * inject enInjectionRate (one of them > 0; both <= 0 turns it off). */
int cup_set_spectral_forcing(struct cup_handle* h, double turbKinEn_target, double enInjectionRate);
/* One SpectralForcing application to the current velocity (operator by
 * operator); stats = totalKinEn, largeModesKinEn, viscousDissip,
 * totalDissipRate, injectionRate, lIntegral (forcingData.dat columns). */
int cup_spectral_forcing(struct cup_handle* h, double dt, double stats[6]);
/* The stats of the last forcing application. */
int cup_get_forcing_stats(struct cup_handle* h, double stats[6]);

/* Test hook for the halo staging (restates tests/cubismup3d/TestBoundaries.cpp):
 * out(x) = f(x - d) through the same periodic plane-streaming TMA path the
 * stencil kernels use, halo g in {1, 2}. f, out: device or host FP64 arrays. */
int cup_debug_shift(struct cup_handle* h, const double* f, double* out, int g, int dx, int dy, int dz, int where);

/* Allocation-free findMaxU: max over n cells of max(|u+uinf0|, |v+uinf1|, |w+uinf2|)
 * for caller-owned device arrays u, v, w (FP64), written to the device double
 * *umax_dev on `stream` (a cudaStream_t; NULL = the legacy default stream); the
 * call is asynchronous. It has no counterpart in the reference. It exists for
 * callers that cannot call cudaMalloc: code whose device memory all comes from
 * another allocator or a budget fixed up front (a framework's caching pool, a
 * long-running service), and loops that must not allocate once running, since
 * cudaMalloc can synchronise the device and can fail late. It allocates
 * nothing: its per-block partial maxima live in a fixed 32 KiB array inside the
 * library (4096 partials, each over at most 65536 cells), which every GPU that
 * loads the library keeps until exit; n above 2^28 cells is rejected with
 * CUP_ERR_ARG. A NaN anywhere in the field makes the result NaN (the handle
 * path reports the same field as CUP_ERR_NONFINITE). Failures return
 * CUP_ERR_ARG or CUP_ERR_CUDA with the reason on stderr (there is no handle for
 * cup_last_error). The first call on a device (and in each new context on it,
 * e.g. after cudaDeviceReset) looks up that array's device address with the
 * device current; make that first call before any stream capture. All calls
 * share the array, so calls that overlap on the GPU (other streams, other host
 * threads) race; every slot a call reads is written by the same call first, so
 * nothing needs clearing between calls. */
int cup_max_velocity_noalloc(const double* u, const double* v, const double* w, long long n,
                             const double uinf[3], double* umax_dev, void* stream);

/* FP32_DC: relative residuals |r| / |b| (null-mode parts excluded) at each
 * check of the last defect-correction solve, check 0 being the warm-started
 * residual before the first FP32 correction; *n_checks = entries written. */
int cup_dc_history(struct cup_handle* h, double* out, int n, int* n_checks);

/* ---- profiling (the reference's Profiler regions, SimulationData.cpp:293-305,
 * as CUDA-event ranges per kernel) ---- */
/* Turns per-kernel CUDA-event timing on or off (off by default; no host sync while on). */
int cup_profile_enable(struct cup_handle* h, int on);
/* Writes {"kernel": {"count": n, "ms": total, "work_count": m, "work_ms": t}, ...} as JSON into buf:
 * all launches, and those that did the pass's work (at least a quarter of the
 * longest launch of that kernel; the kernels of a converged defect-correction
 * loop's later solves exit at entry). reset != 0 clears the records. */
int cup_profile_report(struct cup_handle* h, char* buf, size_t len, int reset);
/* Number of kernels this handle has launched so far. */
int cup_launch_count(const struct cup_handle* h, long long* n);

#ifdef __cplusplus
}
#endif

#endif /* CUP_B200_H */
