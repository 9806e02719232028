// The reference's own operators, driven on one process: the SimulationData,
// grid and operator objects of the reference, built from its headers and its
// operator sources (ref_advect.cpp, ref_rhs.cpp, ref_proj.cpp, ref_pois*.cpp
// compile them unmodified), plus definitions for what those sources declare
// but this build leaves out (the rest of SimulationData, the obstacle classes,
// the non-periodic Poisson solvers: never reached on the periodic path without
// obstacles). Test infrastructure of the oracle only: it checks the oracle's
// restatement against the reference's arithmetic.
//
// C interface (fields are FP64 global arrays [z][y][x], x fastest):
//   ref_create(nx, ny, nz, maxextent, nu, uinf[3]) -> handle
//   ref_set_field / ref_get_field(h, which, f): 0 u, 1 v, 2 w, 3 p, 4 chi,
//     5 tmpU, 6 tmpV, 7 tmpW (the FluidElement members)
//   ref_operator(h, name, dt): "AdvectionDiffusion", "PressureRHS",
//     "PressureProjection" (the reference's operator() on the grid)
//   ref_get_rhs(h, f): the Poisson buffer after PressureRHS, in the global
//     layout
//   ref_destroy(h)
#define CUP_NO_MACROS_HEADER
#include <cstring>
#include <stdexcept>
#include <string>

#include "operators/AdvectionDiffusion.h"
#include "operators/PressureProjection.h"
#include "operators/PressureRHS.h"
#include "obstacles/ObstacleVector.h"
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

// ---- obstacle classes: an empty ObstacleVector (no obstacle is added) ----
[[noreturn]] static void not_here(const char* what) {
  throw std::logic_error(std::string(what) + " is not part of the periodic path without obstacles");
}
void Obstacle::_writeComputedVelToFile() { not_here("Obstacle::_writeComputedVelToFile"); }
void Obstacle::_writeDiagForcesToFile() { not_here("Obstacle::_writeDiagForcesToFile"); }
void Obstacle::_writeSurfForcesToFile() { not_here("Obstacle::_writeSurfForcesToFile"); }
void Obstacle::Accept(ObstacleVisitor*) { not_here("Obstacle::Accept"); }
void Obstacle::computeVelocities() { not_here("Obstacle::computeVelocities"); }
void Obstacle::computeForces() { not_here("Obstacle::computeForces"); }
void Obstacle::update() { not_here("Obstacle::update"); }
void Obstacle::save(std::string) { not_here("Obstacle::save"); }
void Obstacle::restart(std::string) { not_here("Obstacle::restart"); }
void Obstacle::create() { not_here("Obstacle::create"); }
void Obstacle::finalize() { not_here("Obstacle::finalize"); }
std::array<double, 3> Obstacle::getTranslationVelocity() const { not_here("Obstacle::getTranslationVelocity"); }
std::array<double, 3> Obstacle::getAngularVelocity() const { not_here("Obstacle::getAngularVelocity"); }
std::array<double, 3> Obstacle::getCenterOfMass() const { not_here("Obstacle::getCenterOfMass"); }
void ObstacleVector::computeVelocities() {}
void ObstacleVector::update() {}
void ObstacleVector::restart(std::string) {}
void ObstacleVector::save(std::string) {}
void ObstacleVector::computeForces() {}
void ObstacleVector::create() {}
void ObstacleVector::finalize() {}
void ObstacleVector::Accept(ObstacleVisitor* v) {
  for (auto& o : obstacles) o->Accept(v);
}
Real ObstacleVector::getD() const { return 0; }

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

void* ref_create(int nx, int ny, int nz, double maxextent, double nu, const double* uinf) {
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
    s.extent = {nx * h, ny * h, nz * h};
    s.nu = nu;
    for (int d = 0; d < 3; ++d) s.uinf[d] = uinf[d];
    s.BCx_flag = s.BCy_flag = s.BCz_flag = periodic;
    s.bUseFourierBC = true;
    s.obstacle_vector = new ObstacleVector(s);
    // the operators of the periodic pipeline (source/Simulation.cpp:307-401);
    // PressureProjection's constructor makes the Poisson solver
    R->proj = new PressureProjection(s);
    R->advect = new AdvectionDiffusion(s);
    R->rhs = new PressureRHS(s);
    s.pipeline = {R->advect, R->rhs, R->proj};
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

int ref_operator(void* h, const char* name, double dt) {
  RefSim* R = static_cast<RefSim*>(h);
  try {
    R->sim.dt = dt;
    const std::string n(name);
    if (n == "AdvectionDiffusion") (*R->advect)(dt);
    else if (n == "PressureRHS") (*R->rhs)(dt);
    else if (n == "PressureProjection") (*R->proj)(dt);
    else return 1;
    return 0;
  } catch (const std::exception& e) {
    fprintf(stderr, "ref_operator %s: %s\n", name, e.what());
    return 2;
  }
}

}  // extern "C"
