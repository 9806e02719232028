// C++ host facade of the B200-native periodic fractional step, mirroring the
// reference's operator/plugin interface for the hot path:
//
//   class Operator { Operator(SimulationData&); virtual void operator()(double dt) = 0;
//                    virtual std::string getName() = 0; }      (source/operators/Operator.h:16-177)
//   SimulationData with the pipeline and the pressure solver      (source/SimulationData.h:46-179)
//   Simulation::setupOperators / calcMaxTimestep / timestep / run (source/Simulation.cpp:307-623)
//   PoissonSolverPeriodic::solve                                  (source/poisson/PoissonSolverPeriodic.cpp:129-146)
//   FluidGrid of FluidBlocks (16^3 FluidElement blocks, data[z][y][x]) (source/Definitions.h:39-167)
//
// Every operator forwards to one call of the C ABI in include/cup_b200.h; the
// device owns the fields. Where the reference aborts (SimulationData.cpp:180-226,
// Operator.h:40-46) this facade throws: std::invalid_argument for bad input,
// std::runtime_error (with the library's message) otherwise.
#pragma once

#include <array>
#include <cmath>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cup_b200.h"

namespace cubismup3d {

typedef double Real;

inline void cup_check(int rc, cup_handle* h, const char* what) {
  if (rc == CUP_OK) return;
  std::string msg = std::string(what) + ": " + (h ? cup_last_error(h) : "invalid arguments");
  if (rc == CUP_ERR_ARG) throw std::invalid_argument(msg);
  throw std::runtime_error(msg + " (status " + std::to_string(rc) + ")");
}

// FluidElement (source/Definitions.h:39-52): 8 Reals per cell.
struct FluidElement {
  Real chi = 0, u = 0, v = 0, w = 0, p = 0, tmpU = 0, tmpV = 0, tmpW = 0;
};

// BaseBlock<FluidElement> (source/Definitions.h:102-167): 16^3 cells, data[z][y][x].
struct FluidBlock {
  static constexpr int BS = 16, sizeX = BS, sizeY = BS, sizeZ = BS;
  FluidElement data[sizeZ][sizeY][sizeX];
  FluidElement& operator()(int ix, int iy = 0, int iz = 0) { return data[iz][iy][ix]; }
  const FluidElement& operator()(int ix, int iy = 0, int iz = 0) const { return data[iz][iy][ix]; }
};

// The subset of Cubism's BlockInfo the operators use.
struct BlockInfo {
  int blockID;
  std::array<int, 3> index;
  std::array<Real, 3> origin;
  Real h_gridpoint;
  FluidBlock* ptrBlock;
  void pos(Real p[3], int ix, int iy, int iz) const {
    p[0] = origin[0] + h_gridpoint * (ix + 0.5);
    p[1] = origin[1] + h_gridpoint * (iy + 0.5);
    p[2] = origin[2] + h_gridpoint * (iz + 0.5);
  }
};

// Host mirror of the device fields as a grid of FluidBlocks. download() copies
// u, v, w, p, chi from the device; upload() writes u, v, w back.
class FluidGrid {
 public:
  FluidGrid(cup_handle* h, std::array<int, 3> bpd, Real hgrid) : h_(h), bpd_(bpd), hgrid_(hgrid) {
    const int nb = bpd[0] * bpd[1] * bpd[2];
    blocks_.resize(nb);
    infos_.resize(nb);
    for (int bz = 0, id = 0; bz < bpd[2]; ++bz)
      for (int by = 0; by < bpd[1]; ++by)
        for (int bx = 0; bx < bpd[0]; ++bx, ++id)
          infos_[id] = BlockInfo{id, {bx, by, bz}, {bx * 16 * hgrid, by * 16 * hgrid, bz * 16 * hgrid}, hgrid,
                                 &blocks_[id]};
  }
  const std::vector<BlockInfo>& getBlocksInfo() const { return infos_; }
  int getBlocksPerDimension(int d) const { return bpd_[d]; }
  size_t cells() const { return (size_t)bpd_[0] * bpd_[1] * bpd_[2] * 4096; }

  void download() {
    std::vector<double> f[5];
    for (auto& a : f) a.resize(cells());
    cup_check(cup_get_velocity(h_, f[0].data(), f[1].data(), f[2].data(), CUP_WHERE_HOST), h_, "download");
    cup_check(cup_get_pressure(h_, f[3].data(), CUP_WHERE_HOST), h_, "download");
    cup_check(cup_get_chi(h_, f[4].data(), CUP_WHERE_HOST), h_, "download");
    scatter([&](FluidElement& e, size_t g) {
      e.u = f[0][g];
      e.v = f[1][g];
      e.w = f[2][g];
      e.p = f[3][g];
      e.chi = f[4][g];
    });
  }
  void upload() {
    std::vector<double> f[3];
    for (auto& a : f) a.resize(cells());
    scatter([&](FluidElement& e, size_t g) {
      f[0][g] = e.u;
      f[1][g] = e.v;
      f[2][g] = e.w;
    });
    cup_check(cup_set_velocity(h_, f[0].data(), f[1].data(), f[2].data(), CUP_WHERE_HOST), h_, "upload");
  }

 private:
  template <class F>
  void scatter(F&& f) {
    const int nx = bpd_[0] * 16, ny = bpd_[1] * 16;
    for (auto& info : infos_)
      for (int iz = 0; iz < 16; ++iz)
        for (int iy = 0; iy < 16; ++iy)
          for (int ix = 0; ix < 16; ++ix) {
            const size_t g = ((size_t)(info.index[2] * 16 + iz) * ny + (info.index[1] * 16 + iy)) * nx +
                             (info.index[0] * 16 + ix);
            f((*info.ptrBlock)(ix, iy, iz), g);
          }
  }
  cup_handle* h_;
  std::array<int, 3> bpd_;
  Real hgrid_;
  std::vector<FluidBlock> blocks_;
  std::vector<BlockInfo> infos_;
};

class Operator;
class PoissonSolver;

struct SimulationData {
  // grid
  int bpdx = -1, bpdy = -1, bpdz = -1;
  Real maxextent = 1;
  Real hmin = 0, hmax = 0, hmean = 0;
  // flow
  std::array<Real, 3> uinf = {{0, 0, 0}};
  double nu = 0, CFL = 0, lambda = -1, DLM = 1;  // struct defaults of the reference
  int rampup = 100;
  bool bImplicitPenalization = false;
  // status
  int step = 0, nsteps = 0;
  double time = 0, endTime = 0, dt = 0;
  int freqDiagnostics = 0;  // ComputeDissipation every this many steps (0: off)
  double turbKinEn_target = 0, enInjectionRate = 0;  // SpectralForcing (SimulationData.cpp:60-66)
  // B200 form
  int precision = CUP_PREC_FP64;
  int scheme = CUP_SCHEME_REF;
  double dc_tol = 1e-10;
  int dc_max_iter = 4, dc_min_iter = 1;
  int device = 0;
  // owned state
  cup_handle* handle = nullptr;
  bool has_obstacle = false;  // obstacle_vector->nObstacles() > 0
  std::unique_ptr<FluidGrid> grid;
  std::vector<Operator*> pipeline;
  PoissonSolver* pressureSolver = nullptr;

  void setCells(int nx, int ny, int nz) {  // SimulationData::setCells (SimulationData.cpp:280-291)
    if (nx % 16 || ny % 16 || nz % 16)
      throw std::invalid_argument("Number of cells must be multiple of block size * number of processes.");
    bpdx = nx / 16;
    bpdy = ny / 16;
    bpdz = nz / 16;
  }
  const std::vector<BlockInfo>& vInfo() const { return grid->getBlocksInfo(); }
  inline ~SimulationData();
};

class Operator {
 protected:
  SimulationData& sim;

 public:
  explicit Operator(SimulationData& s) : sim(s) {}
  virtual ~Operator() = default;
  virtual void operator()(const double dt) = 0;
  virtual std::string getName() = 0;
};

// PoissonSolver (source/poisson/PoissonSolver.h:22-122): the public buffer
// contract `data`, stridex/y/z, data_size, _offset / _offset_ext / _dest,
// reset() and _fftw2cub(). `data` is the handle's FP64 device array: device
// code (or cudaMemcpy, or cup_set_rhs for a host array) writes the
// h^3-premultiplied RHS at data[_dest(_offset_ext(info), iz, iy, ix)] before
// solve(), as the reference's kernels write solver->data.
class PoissonSolver {
 public:
  size_t stridez = 0, stridey = 0, stridex = 0, data_size = 0;
  Real* data = nullptr;
  virtual ~PoissonSolver() = default;
  virtual void solve() = 0;
  virtual void reset() const = 0;
  // The solve writes the solution into the pressure itself (the last inverse
  // transform pass), so the copy back into the blocks has nothing left to do.
  void _fftw2cub() const {}
  size_t _offset(const BlockInfo& info) const {
    return stridez * (size_t)info.index[2] * FluidBlock::sizeZ + stridey * (size_t)info.index[1] * FluidBlock::sizeY +
           stridex * (size_t)info.index[0] * FluidBlock::sizeX;
  }
  size_t _offset_ext(const BlockInfo& info) const { return _offset(info); }
  size_t _dest(const size_t offset, const int z, const int y, const int x) const {
    return offset + stridez * z + stridey * y + stridex * x;
  }
};

class PoissonSolverPeriodic : public PoissonSolver {
  SimulationData& sim;

 public:
  inline explicit PoissonSolverPeriodic(SimulationData& s);
  cup_solve_stats last{};
  void solve() override { cup_check(cup_poisson_solve(sim.handle, &last), sim.handle, "PoissonSolverPeriodic::solve"); }
  void reset() const override { cup_check(cup_poisson_reset(sim.handle), sim.handle, "PoissonSolver::reset"); }
};

// CreateObstacles (source/operators/ObstaclesCreate.cpp:444-540): moves a
// sphere that is not at rest in the frame by dt (transVel + uinf) and rebuilds
// its chi; nothing otherwise.
class CreateObstacles : public Operator {
 public:
  using Operator::Operator;
  void operator()(const double dt) override {
    cup_check(cup_create_obstacles(sim.handle, dt), sim.handle, "CreateObstacles");
  }
  std::string getName() override { return "CreateObstacles"; }
};

// UpdateObstacles (source/operators/ObstaclesUpdate.cpp:202-236): the free
// dofs' velocities from the fluid momentum balance of
// Obstacle::computeVelocities (source/obstacles/Obstacle.cpp:153-264); forced
// dofs keep their imposed velocity.
class UpdateObstacles : public Operator {
 public:
  using Operator::Operator;
  void operator()(const double dt) override {
    cup_check(cup_update_obstacles(sim.handle, dt), sim.handle, "UpdateObstacles");
  }
  std::string getName() override { return "UpdateObstacles"; }
};

class AdvectionDiffusion : public Operator {
 public:
  using Operator::Operator;
  void operator()(const double dt) override {
    cup_check(cup_advect_diffuse(sim.handle, dt), sim.handle, "AdvectionDiffusion");
  }
  std::string getName() override { return "AdvectionDiffusion"; }
};

// SpectralForcing (source/spectralOperators/SpectralForcing.cpp:23-86): raises the
// energy of the band 0 < k^2 <= 4 to meet turbKinEn_target or enInjectionRate.
class SpectralForcing : public Operator {
 public:
  using Operator::Operator;
  std::array<double, 6> stats{};  // totalKinEn, largeModesKinEn, viscousDissip, totalDissipRate, injectionRate, lIntegral
  void operator()(const double dt) override {
    cup_check(cup_spectral_forcing(sim.handle, dt, stats.data()), sim.handle, "SpectralForcing");
  }
  std::string getName() override { return "SpectralForcing"; }
};

class PressureRHS : public Operator {
 public:
  using Operator::Operator;
  void operator()(const double dt) override { cup_check(cup_pressure_rhs(sim.handle, dt), sim.handle, "PressureRHS"); }
  std::string getName() override { return "PressureRHS"; }
};

class PressureProjection : public Operator {
 public:
  using Operator::Operator;
  void operator()(const double dt) override {
    sim.pressureSolver->solve();
    sim.pressureSolver->_fftw2cub();
    cup_check(cup_grad_correct(sim.handle, dt), sim.handle, "PressureProjection");
  }
  std::string getName() override { return "PressureProjection"; }
};

class Penalization : public Operator {
 public:
  using Operator::Operator;
  std::array<double, 6> force_torque{};
  void operator()(const double dt) override {
    cup_check(cup_penalize(sim.handle, dt, force_torque.data()), sim.handle, "Penalization");
  }
  std::string getName() override { return "Penalization"; }
};

// ComputeForces (source/operators/FluidSolidForces.cpp:200-222) after
// Penalization: the surface forces of the sphere on the final velocity and
// pressure (cup_compute_forces), appended every step to
// forceValues_surface_0.dat and powerValues_surface_0.dat in the format of
// Obstacle::_writeSurfForcesToFile (source/obstacles/Obstacle.cpp:518-556).
// Nothing without an obstacle.
class ComputeForces : public Operator {
 public:
  using Operator::Operator;
  // surfForce[3], presForce[3], viscForce[3], surfTorque[3], gamma[3], drag, thrust, Pout, PoutBnd,
  // defPower, defPowerBnd, pLocom, Pthrust, Pdrag, EffPDef, EffPDefBnd, mass
  std::array<double, 27> last{};
  void operator()(const double) override {
    if (!sim.has_obstacle) return;
    cup_check(cup_compute_forces(sim.handle, last.data()), sim.handle, "ComputeForces");
    const double* q = last.data();
    std::FILE* f = std::fopen("forceValues_surface_0.dat", "a");
    if (!f) throw std::runtime_error("ComputeForces: cannot open forceValues_surface_0.dat");
    if (sim.step == 0)
      std::fprintf(f, "step\ttime\tmass\tforce_x\tforce_y\tforce_z\ttorque_x\ttorque_y\ttorque_z\tpresF_x\t"
                      "presF_y\tpresF_z\tviscF_x\tviscF_y\tviscF_z\tgamma_x\tgamma_y\tgamma_z\tdrag\tthrust\n");
    std::fprintf(f, "%d\t%.7e\t%.7e", sim.step, sim.time, q[26]);
    for (int k : {0, 1, 2, 9, 10, 11, 3, 4, 5, 6, 7, 8, 12, 13, 14, 15, 16}) std::fprintf(f, "\t%.7e", q[k]);
    std::fprintf(f, "\n");
    std::fclose(f);
    f = std::fopen("powerValues_surface_0.dat", "a");
    if (!f) throw std::runtime_error("ComputeForces: cannot open powerValues_surface_0.dat");
    if (sim.step == 0)
      std::fprintf(f, "step\ttime\tPthrust\tPdrag\tPout\tpDef\tetaPDef\tpLocom\tPoutBnd\tdefPowerBnd\tetaPDefBnd\n");
    std::fprintf(f, "%d\t%.7e\t%.7e\t%.7e\t%.7e\t%.7e\t%.7e\t%.7e\t%.7e\t%.7e\t%.7e\n", sim.step, sim.time, q[22],
                 q[23], q[17], -q[19], q[24], q[21], q[18], -q[20], q[25]);
    std::fclose(f);
  }
  std::string getName() override { return "ComputeForces"; }
};

// ComputeDissipation (source/operators/ComputeDissipation.cpp:119-177): every
// freqDiagnostics steps, the 20 sums of the current fields appended to
// diagnostics.dat in the reference's format (header at step 0).
class ComputeDissipation : public Operator {
 public:
  using Operator::Operator;
  std::array<double, 20> last{};
  void operator()(const double) override {
    if (sim.freqDiagnostics == 0 || sim.step % sim.freqDiagnostics) return;
    cup_check(cup_compute_dissipation(sim.handle, last.data()), sim.handle, "ComputeDissipation");
    std::FILE* f = std::fopen("diagnostics.dat", "a");
    if (!f) throw std::runtime_error("ComputeDissipation: cannot open diagnostics.dat");
    if (sim.step == 0)
      std::fprintf(f, "step_id time circ_x circ_y circ_y linImp_x linImp_y linImp_z linMom_x linMom_y linMom_z "
                      "angImp_x angImp_y angImp_z angMom_x angMom_y angMom_z presPow viscPow helicity kineticEn "
                      "enstrophy\n");
    std::fprintf(f, "%d %g", sim.step, sim.time);
    for (double x : last) std::fprintf(f, " %g", x);
    std::fprintf(f, "\n");
    std::fclose(f);
  }
  std::string getName() override { return "ComputeDissipation"; }
};

PoissonSolverPeriodic::PoissonSolverPeriodic(SimulationData& s) : sim(s) {
  size_t st[3] = {0, 0, 0};
  cup_check(cup_poisson_buffer(sim.handle, &data, st, &data_size), sim.handle, "PoissonSolverPeriodic");
  stridex = st[0];
  stridey = st[1];
  stridez = st[2];
}

SimulationData::~SimulationData() {
  while (!pipeline.empty()) {
    delete pipeline.back();
    pipeline.pop_back();
  }
  delete pressureSolver;
  if (handle) cup_destroy(handle);
}

// Sphere arguments (source/obstacles/Obstacle.h:60-75 + SphereArguments).
struct SphereArguments {
  double radius = 0.1;
  std::array<double, 3> position = {{0.5, 0.5, 0.5}};
  std::array<double, 3> enforcedVelocity = {{0, 0, 0}};
  std::array<bool, 3> bForcedInSimFrame = {{true, true, true}};
  std::array<bool, 3> bFixFrameOfRef = {{false, false, false}};
};

class Simulation {
 public:
  SimulationData sim;

  // Simulation(const SimulationData&) (source/Simulation.cpp:53-64)
  explicit Simulation(const SimulationData& cfg) {
    copy_params(cfg);
    cup_config c{};
    c.bpdx = sim.bpdx;
    c.bpdy = sim.bpdy;
    c.bpdz = sim.bpdz;
    c.maxextent = sim.maxextent;
    c.nu = sim.nu;
    c.CFL = sim.CFL;
    c.lambda = sim.lambda;
    c.DLM = sim.DLM;
    for (int d = 0; d < 3; ++d) c.uinf[d] = sim.uinf[d];
    c.rampup = sim.rampup;
    c.bImplicitPenalization = sim.bImplicitPenalization;
    c.precision = sim.precision;
    c.scheme = sim.scheme;
    c.dc_tol = sim.dc_tol;
    c.dc_max_iter = sim.dc_max_iter;
    c.dc_min_iter = sim.dc_min_iter;
    c.device = sim.device;
    if (!(sim.lambda > 0 || sim.DLM > 0)) throw std::invalid_argument("need lambda > 0 or DLM > 0");
    cup_check(cup_create(&c, &sim.handle), nullptr, "cup_create");
    int cells[3];
    double h = 0;
    cup_get_dims(sim.handle, cells, &h);
    sim.hmin = sim.hmax = sim.hmean = h;
    sim.grid.reset(new FluidGrid(sim.handle, {sim.bpdx, sim.bpdy, sim.bpdz}, h));
    sim.pressureSolver = new PoissonSolverPeriodic(sim);
    setupOperators();
  }
  Simulation(const Simulation&) = delete;

  // The periodic hot-path pipeline of Simulation::setupOperators (source/Simulation.cpp:307-401).
  void setupOperators() {
    for (auto* op : sim.pipeline) delete op;
    sim.pipeline.clear();
    sim.pipeline.push_back(new CreateObstacles(sim));
    sim.pipeline.push_back(new AdvectionDiffusion(sim));
    if (sim.turbKinEn_target > 0 || sim.enInjectionRate > 0) {
      if (sim.turbKinEn_target > 0 && sim.enInjectionRate > 0)
        throw std::invalid_argument("give either turbKinEn_target or enInjectionRate, not both");
      cup_check(cup_set_spectral_forcing(sim.handle, sim.turbKinEn_target, sim.enInjectionRate), sim.handle,
                "SpectralForcing");
      sim.pipeline.push_back(new SpectralForcing(sim));
    }
    sim.pipeline.push_back(new PressureRHS(sim));
    sim.pipeline.push_back(new PressureProjection(sim));
    sim.pipeline.push_back(new UpdateObstacles(sim));
    sim.pipeline.push_back(new Penalization(sim));
    sim.pipeline.push_back(new ComputeForces(sim));
    sim.pipeline.push_back(new ComputeDissipation(sim));
  }

  void add_obstacle(const SphereArguments& a) {
    cup_sphere s{};
    s.radius = a.radius;
    for (int d = 0; d < 3; ++d) {
      s.position[d] = a.position[d];
      s.enforcedVelocity[d] = a.enforcedVelocity[d];
      s.bForcedInSimFrame[d] = a.bForcedInSimFrame[d];
      s.bFixFrameOfRef[d] = a.bFixFrameOfRef[d];
    }
    cup_check(cup_add_sphere(sim.handle, &s), sim.handle, "add_obstacle");
    sim.has_obstacle = true;
  }

  double calcMaxTimestep() {
    cup_check(cup_calc_max_timestep(sim.handle, &sim.dt), sim.handle, "calcMaxTimestep");
    return sim.dt;
  }

  // Simulation::timestep (source/Simulation.cpp:593-623): runs the pipeline
  // operator by operator; returns true when nsteps or endTime is reached.
  bool timestep(const double dt) {
    for (auto* op : sim.pipeline) (*op)(dt);
    sim.step++;
    sim.time += dt;
    cup_check(cup_set_clock(sim.handle, sim.step, sim.time), sim.handle, "timestep");
    return (sim.endTime > 0 && sim.time > sim.endTime) || (sim.nsteps != 0 && sim.step >= sim.nsteps);
  }

  // Simulation::run (source/Simulation.cpp:582-591)
  void run() {
    for (;;) {
      const double dt = calcMaxTimestep();
      if (timestep(dt)) break;
    }
  }

 private:
  void copy_params(const SimulationData& c) {
    sim.bpdx = c.bpdx;
    sim.bpdy = c.bpdy;
    sim.bpdz = c.bpdz;
    sim.maxextent = c.maxextent;
    sim.uinf = c.uinf;
    sim.nu = c.nu;
    sim.CFL = c.CFL;
    sim.lambda = c.lambda;
    sim.DLM = c.DLM;
    sim.rampup = c.rampup;
    sim.bImplicitPenalization = c.bImplicitPenalization;
    sim.nsteps = c.nsteps;
    sim.endTime = c.endTime;
    sim.freqDiagnostics = c.freqDiagnostics;
    sim.turbKinEn_target = c.turbKinEn_target;
    sim.enInjectionRate = c.enInjectionRate;
    sim.precision = c.precision;
    sim.scheme = c.scheme;
    sim.dc_tol = c.dc_tol;
    sim.dc_max_iter = c.dc_max_iter;
    sim.dc_min_iter = c.dc_min_iter;
    sim.device = c.device;
  }
};

}  // namespace cubismup3d
