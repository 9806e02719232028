// Drives the periodic pipeline through the C++ Operator facade
// (cubismup_3d_b200/cpp/cubismup3d.hpp) the way Simulation::run does
// (source/Simulation.cpp:582-623): Taylor-Green at n^3, nsteps of
// calcMaxTimestep + operator-by-operator timestep, then writes u, v, w
// (FP64, [z][y][x]) and the dt sequence to the output file.
// Usage: tg_driver <n> <nsteps> <scheme 0|1> <out.bin>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cubismup3d.hpp"

int main(int argc, char** argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s n nsteps scheme out.bin\n", argv[0]);
    return 2;
  }
  const int n = atoi(argv[1]), nsteps = atoi(argv[2]), scheme = atoi(argv[3]);
  using namespace cubismup3d;
  try {
    SimulationData sd;
    sd.setCells(n, n, n);
    sd.maxextent = 2 * M_PI;
    sd.nu = 0.01;
    sd.CFL = 0.5;
    sd.rampup = 3;
    sd.DLM = 0;
    sd.lambda = 1;
    sd.nsteps = nsteps;
    sd.scheme = scheme;
    Simulation S(sd);
    const double h = S.sim.hmin;
    // Taylor-Green initial condition through the FluidGrid of FluidBlocks
    for (const BlockInfo& info : S.sim.vInfo())
      for (int iz = 0; iz < 16; ++iz)
        for (int iy = 0; iy < 16; ++iy)
          for (int ix = 0; ix < 16; ++ix) {
            Real p[3];
            info.pos(p, ix, iy, iz);
            FluidElement& e = (*info.ptrBlock)(ix, iy, iz);
            e.u = std::sin(p[0]) * std::cos(p[1]) * std::cos(p[2]);
            e.v = -std::cos(p[0]) * std::sin(p[1]) * std::cos(p[2]);
            e.w = 0;
          }
    S.sim.grid->upload();
    std::vector<double> dts;
    for (;;) {
      const double dt = S.calcMaxTimestep();
      dts.push_back(dt);
      if (S.timestep(dt)) break;
    }
    std::vector<double> f[3];
    for (auto& a : f) a.resize((size_t)n * n * n);
    cup_check(cup_get_velocity(S.sim.handle, f[0].data(), f[1].data(), f[2].data(), CUP_WHERE_HOST), S.sim.handle,
              "get_velocity");
    FILE* fp = fopen(argv[4], "wb");
    if (!fp) return 3;
    for (auto& a : f) fwrite(a.data(), sizeof(double), a.size(), fp);
    fwrite(dts.data(), sizeof(double), dts.size(), fp);
    fclose(fp);
    printf("%zu steps, t=%.6f\n", dts.size(), S.sim.time);
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
