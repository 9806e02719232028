// The reference's own operators, driven on one process: the SimulationData,
// grid and operator objects of the reference, built from its headers and its
// operator and obstacle sources (the ref_*.cpp files of this directory compile
// them unmodified), plus definitions for what those sources declare but this
// build leaves out (the rest of SimulationData, the non-periodic Poisson
// solvers: never reached on the uniform periodic path). Test infrastructure of
// the oracle only: it checks the oracle's restatement against the reference's
// arithmetic.
//
// C interface (fields are FP64 global arrays [z][y][x], x fastest):
//   ref_create(nx, ny, nz, maxextent, nu, uinf[3]) -> handle
//   ref_set_field / ref_get_field(h, which, f): 0 u, 1 v, 2 w, 3 p, 4 chi,
//     5 tmpU, 6 tmpV, 7 tmpW (the FluidElement members)
//   ref_add_sphere(h, radius, position[3], enforcedVelocity[3], forced[3],
//     fixFrame[3]): a Sphere (source/obstacles/Sphere.cpp) in the obstacle
//     vector, then CreateObstacles(0) as Simulation::setupOperators does
//   ref_operator(h, name, dt): "CreateObstacles", "AdvectionDiffusion",
//     "PressureRHS", "PressureProjection", "UpdateObstacles", "Penalization",
//     "ComputeForces" (the reference's operator() on the grid)
//   ref_obstacle(h, out[48]): the sphere's state (see ref_obstacle)
//   ref_get_rhs(h, f): the Poisson buffer after PressureRHS, in the global
//     layout
//   ref_destroy(h)
#define CUP_NO_MACROS_HEADER
#include <cstring>
#include <stdexcept>
#include <string>

#include "obstacles/ObstacleVector.h"
#include "utils/BufferedLogger.h"
#include "obstacles/Sphere.h"
#include "operators/AdvectionDiffusion.h"
#include "operators/FluidSolidForces.h"
#include "operators/ObstaclesCreate.h"
#include "operators/ObstaclesUpdate.h"
#include "operators/Penalization.h"
#include "operators/PressureProjection.h"
#include "operators/PressureRHS.h"
#include "poisson/PoissonSolverMixed.h"
#include "poisson/PoissonSolverPeriodic.h"
#include "poisson/PoissonSolverUnbounded.h"

namespace cubismup3d {

// ---- SimulationData (the members of source/SimulationData.cpp this path reads
// are plain fields; the constructor sets the communicator only) ----
SimulationData::SimulationData(MPI_Comm mpicomm) : app_comm(mpicomm) {}
SimulationData::~SimulationData() {
  for (Operator* op : pipeline) delete op;
  delete pressureSolver;
  delete obstacle_vector;
  delete grid;
}
void SimulationData::startProfiler(std::string) const {}
void SimulationData::stopProfiler() const {}

[[noreturn]] static void not_here(const char* what) {
  throw std::logic_error(std::string(what) + " is not part of the uniform periodic path");
}

// ---- the non-periodic Poisson solvers PressureProjection can select ----
PoissonSolverUnbounded::PoissonSolverUnbounded(SimulationData& s) : PoissonSolver(s) {
  not_here("PoissonSolverUnbounded");
}
PoissonSolverUnbounded::~PoissonSolverUnbounded() {}
void PoissonSolverUnbounded::solve() { not_here("PoissonSolverUnbounded::solve"); }
void PoissonSolverUnbounded::reset() const { not_here("PoissonSolverUnbounded::reset"); }
PoissonSolverMixed::PoissonSolverMixed(SimulationData& s) : PoissonSolver(s) { not_here("PoissonSolverMixed"); }
PoissonSolverMixed::~PoissonSolverMixed() {}
void PoissonSolverMixed::solve() { not_here("PoissonSolverMixed::solve"); }

}  // namespace cubismup3d

using namespace cubismup3d;

namespace {

struct RefSim {
  SimulationData sim{MPI_COMM_WORLD};
  int nx = 0, ny = 0, nz = 0;
  AdvectionDiffusion* advect = nullptr;
  PressureRHS* rhs = nullptr;
  PressureProjection* proj = nullptr;
  CreateObstacles* create = nullptr;
  UpdateObstacles* update = nullptr;
  Penalization* penal = nullptr;
  ComputeForces* forces = nullptr;
};

Real& member(FluidElement& e, int which) {
  switch (which) {
    case 0: return e.u;
    case 1: return e.v;
    case 2: return e.w;
    case 3: return e.p;
    case 4: return e.chi;
    case 5: return e.tmpU;
    case 6: return e.tmpV;
    default: return e.tmpW;
  }
}

template <class F>
void for_cells(RefSim* R, F&& f) {
  const int S = FluidBlock::sizeX;
  for (const cubism::BlockInfo& I : R->sim.grid->getBlocksInfo()) {
    FluidBlock& b = *(FluidBlock*)I.ptrBlock;
    for (int iz = 0; iz < S; ++iz)
      for (int iy = 0; iy < S; ++iy)
        for (int ix = 0; ix < S; ++ix) {
          const size_t g = ((size_t)(I.index[2] * S + iz) * R->ny + (I.index[1] * S + iy)) * R->nx +
                           (I.index[0] * S + ix);
          f(b(ix, iy, iz), g, I, ix, iy, iz);
        }
  }
}

}  // namespace

extern "C" {

void* ref_create(int nx, int ny, int nz, double maxextent, double nu, const double* uinf, double lambda,
                 int implicit) {
  try {
    RefSim* R = new RefSim();
    R->nx = nx, R->ny = ny, R->nz = nz;
    SimulationData& s = R->sim;
    s.rank = 0, s.nprocs = 1, s.nprocsx = s.nprocsy = s.nprocsz = 1;
    s.bpdx = s.local_bpdx = nx / FluidBlock::sizeX;
    s.bpdy = s.local_bpdy = ny / FluidBlock::sizeY;
    s.bpdz = s.local_bpdz = nz / FluidBlock::sizeZ;
    s.maxextent = maxextent;
    s.grid = new FluidGridMPI(1, 1, 1, s.bpdx, s.bpdy, s.bpdz, maxextent, MPI_COMM_WORLD);
    const double h = s.grid->getH();
    s.hmin = s.hmax = s.hmean = h;
    // the block extents the obstacles' isTouching reads (Simulation::setupGrid,
    // source/Simulation.cpp:295-304)
    for (const cubism::BlockInfo& I : s.grid->getBlocksInfo()) {
      FluidBlock& b = *(FluidBlock*)I.ptrBlock;
      b.min_pos = I.pos<Real>(0, 0, 0);
      b.max_pos = I.pos<Real>(FluidBlock::sizeX - 1, FluidBlock::sizeY - 1, FluidBlock::sizeZ - 1);
    }
    s.extent = {nx * h, ny * h, nz * h};
    s.nu = nu;
    s.lambda = lambda;
    s.DLM = 0;
    s.bImplicitPenalization = implicit != 0;
    for (int d = 0; d < 3; ++d) s.uinf[d] = uinf[d];
    s.BCx_flag = s.BCy_flag = s.BCz_flag = periodic;
    s.bUseFourierBC = true;
    s.obstacle_vector = new ObstacleVector(s);
    // the operators of the periodic pipeline (source/Simulation.cpp:307-401);
    // PressureProjection's constructor makes the Poisson solver
    R->proj = new PressureProjection(s);
    R->create = new CreateObstacles(s);
    R->advect = new AdvectionDiffusion(s);
    R->rhs = new PressureRHS(s);
    R->update = new UpdateObstacles(s);
    R->penal = new Penalization(s);
    R->forces = new ComputeForces(s);
    s.pipeline = {R->create, R->advect, R->rhs, R->proj, R->update, R->penal, R->forces};
    return R;
  } catch (const std::exception& e) {
    fprintf(stderr, "ref_create: %s\n", e.what());
    return nullptr;
  }
}

void ref_destroy(void* h) { delete static_cast<RefSim*>(h); }

void ref_set_field(void* h, int which, const double* f) {
  for_cells(static_cast<RefSim*>(h),
            [&](FluidElement& e, size_t g, const cubism::BlockInfo&, int, int, int) { member(e, which) = f[g]; });
}

void ref_get_field(void* h, int which, double* f) {
  for_cells(static_cast<RefSim*>(h),
            [&](FluidElement& e, size_t g, const cubism::BlockInfo&, int, int, int) { f[g] = member(e, which); });
}

// The Poisson buffer (solver->data at _offset_ext(info) + stridez iz + stridey iy + stridex ix).
void ref_get_rhs(void* h, double* f) {
  RefSim* R = static_cast<RefSim*>(h);
  PoissonSolver* ps = R->sim.pressureSolver;
  for_cells(R, [&](FluidElement&, size_t g, const cubism::BlockInfo& I, int ix, int iy, int iz) {
    f[g] = ps->data[ps->_offset_ext(I) + ps->stridez * iz + ps->stridey * iy + ps->stridex * ix];
  });
}

int ref_add_sphere(void* h, double radius, const double* position, const double* vel, const int* forced,
                   const int* fix_frame) {
  RefSim* R = static_cast<RefSim*>(h);
  try {
    ObstacleArguments oa;
    oa.length = 2 * radius;
    for (int d = 0; d < 3; ++d) {
      oa.position[d] = position[d];
      oa.enforcedVelocity[d] = vel[d];
      oa.bForcedInSimFrame[d] = forced[d] != 0;
      oa.bFixFrameOfRef[d] = fix_frame[d] != 0;
    }
    R->sim.obstacle_vector->addObstacle(
        std::make_shared<Sphere>(R->sim, ObstacleAndSphereArguments(oa, SphereArguments(radius))));
    (*R->create)(0);  // Simulation::setupOperators creates the obstacles at once
    return 0;
  } catch (const std::exception& e) {
    fprintf(stderr, "ref_add_sphere: %s\n", e.what());
    return 1;
  }
}

// The sphere's state: [0..2] force, [3..5] torque (Penalization), [6..8]
// centerOfMass, [9..11] transVel, [12..14] angVel, [15..17] position, [18..20]
// sim.uinf, [21] mass, then the 22 ComputeForces sums in ObstacleBlock::sumQoI
// order at [22..43], Pthrust, Pdrag, EffPDef, EffPDefBnd at [44..47].
int ref_obstacle(void* h, double* out) {
  RefSim* R = static_cast<RefSim*>(h);
  if (R->sim.obstacle_vector->nObstacles() == 0) return 1;
  const Obstacle& o = *R->sim.obstacle_vector->getObstacleVector()[0];
  for (int d = 0; d < 3; ++d) {
    out[d] = o.force[d];
    out[3 + d] = o.torque[d];
    out[6 + d] = o.centerOfMass[d];
    out[9 + d] = o.transVel[d];
    out[12 + d] = o.angVel[d];
    out[15 + d] = o.position[d];
    out[18 + d] = R->sim.uinf[d];
  }
  out[21] = o.mass;
  const double q[26] = {o.surfForce[0], o.surfForce[1], o.surfForce[2], o.presForce[0], o.presForce[1],
                        o.presForce[2], o.viscForce[0], o.viscForce[1], o.viscForce[2], o.surfTorque[0],
                        o.surfTorque[1], o.surfTorque[2], o.gamma[0], o.gamma[1], o.gamma[2], o.drag, o.thrust,
                        o.Pout, o.PoutBnd, o.defPower, o.defPowerBnd, o.pLocom, o.Pthrust, o.Pdrag, o.EffPDef,
                        o.EffPDefBnd};
  for (int k = 0; k < 26; ++k) out[22 + k] = q[k];
  return 0;
}

// Clock of the step (Simulation::timestep advances it after the pipeline).
void ref_set_clock(void* h, int step, double time, double dt) {
  RefSim* R = static_cast<RefSim*>(h);
  R->sim.step = step, R->sim.time = time, R->sim.dt = dt;
}

int ref_operator(void* h, const char* name, double dt) {
  RefSim* R = static_cast<RefSim*>(h);
  try {
    R->sim.dt = dt;
    const std::string n(name);
    if (n == "CreateObstacles") (*R->create)(dt);
    else if (n == "AdvectionDiffusion") (*R->advect)(dt);
    else if (n == "PressureRHS") (*R->rhs)(dt);
    else if (n == "PressureProjection") (*R->proj)(dt);
    else if (n == "UpdateObstacles") (*R->update)(dt);
    else if (n == "Penalization") (*R->penal)(dt);
    else if (n == "ComputeForces") (*R->forces)(dt);
    else return 1;
    return 0;
  } catch (const std::exception& e) {
    fprintf(stderr, "ref_operator %s: %s\n", name, e.what());
    return 2;
  }
}

// Writes the reference logger's buffered lines (the obstacle's force and
// velocity logs) into the working directory now rather than at exit.
void ref_flush_logs() { cubismup3d::logger.flush(); }

}  // extern "C"
