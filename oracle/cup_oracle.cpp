// ORACLE — test infrastructure only.
//
// A CPU FP64 restatement of CubismUP_3D's fractional-step time step on a
// uniform periodic grid of 16^3-cell blocks. It is the checker for the CUDA
// product path and the timed CPU baseline; the product never links or calls
// it. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it.
//
// Parity status:
//   * periodic halo semantics (Cubism BlockLab, which is not in the reference
//     snapshot) are pinned by a restatement of tests/cubismup3d/TestBoundaries.cpp
//     (see orc_lab_shift and tests/test_oracle.py);
//   * the FFT Poisson solve follows FFTW 3.3.7's published unnormalised DFT
//     definition (third-party, absent here); it is pinned against numpy's
//     pocketfft in tests/test_oracle.py and tests/golden/;
//   * no outputs of the reference itself exist: it cannot be built in this
//     image (MPI, FFTW-MPI, HDF5, GSL and the Cubism sources are absent).
//
// Every kernel cites the reference file:line it restates. Expression order
// follows the reference so that rounding matches where the algorithm does.
// Build: oracle/Makefile (g++ -O3 -march=x86-64-v3 -fopenmp, no -ffast-math,
// -ffp-contract=off so results do not depend on FMA contraction).

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>
#include <omp.h>

namespace {

constexpr int BS = 16;                 // CUP_BLOCK_SIZE (source/Definitions.h:27-29)
typedef double Real;                   // source/Base.h:38-42
constexpr Real EPS = std::numeric_limits<Real>::epsilon();
constexpr int SURFDH = 1;              // source/ObstacleBlock.h:16

struct Dims {
  int nx, ny, nz;
  size_t n() const { return (size_t)nx * ny * nz; }
  size_t idx(int x, int y, int z) const { return ((size_t)z * ny + y) * nx + x; }
  int bpd(int d) const { return (d == 0 ? nx : d == 1 ? ny : nz) / BS; }
  int nblocks() const { return bpd(0) * bpd(1) * bpd(2); }
};

inline int wrap(int i, int n) { i %= n; return i < 0 ? i + n : i; }

// One block of one scalar field plus a g-wide periodic halo, including edges
// and corners (the "tensorial" fill). Replaces Cubism's BlockLab for periodic
// boundaries: ghosts come from the neighbouring blocks with periodic wrap
// (source/operators/Operator.h:112-170, source/Definitions.h:260-378).
struct Lab {
  int g = 1, W = BS + 2;
  std::vector<Real> d;
  void load(const Real* f, const Dims& D, int bx, int by, int bz, int g_) {
    g = g_; W = BS + 2 * g;
    d.resize((size_t)W * W * W);
    const int x0 = bx * BS - g, y0 = by * BS - g, z0 = bz * BS - g;
    for (int k = 0; k < W; ++k) {
      const int z = wrap(z0 + k, D.nz);
      for (int j = 0; j < W; ++j) {
        const int y = wrap(y0 + j, D.ny);
        const Real* row = f + D.idx(0, y, z);
        Real* out = &d[((size_t)k * W + j) * W];
        for (int i = 0; i < W; ++i) out[i] = row[wrap(x0 + i, D.nx)];
      }
    }
  }
  Real operator()(int ix, int iy, int iz) const {
    return d[((size_t)(iz + g) * W + (iy + g)) * W + (ix + g)];
  }
};

template <typename F>
void for_each_block(const Dims& D, F&& f) {
  const int nb = D.nblocks();
  #pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    f(bx, by, bz);
  }
}

// ---------------------------------------------------------------------------
// Complex radix-2 FFT on a contiguous line (unnormalised, FFTW sign
// convention: forward e^{-2 pi i k n/N}, backward e^{+2 pi i k n/N}).
// Twiddles are computed in long double on the host.
struct FFTPlan {
  int n = 0, logn = 0;
  std::vector<std::complex<Real>> tw;  // e^{-2 pi i k/n}, k < n/2
  std::vector<int> rev;
  void init(int n_) {
    n = n_; logn = 0;
    while ((1 << logn) < n) ++logn;
    tw.resize(n / 2 > 0 ? n / 2 : 1);
    for (int k = 0; k < n / 2; ++k) {
      const long double a = -2.0L * 3.141592653589793238462643383279502884L * k / n;
      tw[k] = std::complex<Real>((Real)std::cos(a), (Real)std::sin(a));
    }
    rev.resize(n);
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int b = 0; b < logn; ++b) if (i & (1 << b)) r |= 1 << (logn - 1 - b);
      rev[i] = r;
    }
  }
  void exec(std::complex<Real>* a, int sign) const {
    for (int i = 0; i < n; ++i) if (i < rev[i]) std::swap(a[i], a[rev[i]]);
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len / 2, step = n / len;
      for (int i = 0; i < n; i += len)
        for (int j = 0; j < half; ++j) {
          std::complex<Real> w = tw[j * step];
          if (sign > 0) w = std::conj(w);
          const std::complex<Real> t = w * a[i + j + half];
          a[i + j + half] = a[i + j] - t;
          a[i + j] = a[i + j] + t;
        }
    }
  }
};

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// FFTW-layout buffer of the periodic Poisson solver:
// data[x*stridex + y*stridey + z], stridez = 1, stridey = 2*nz_hat,
// stridex = Ny*2*nz_hat (source/poisson/PoissonSolverPeriodic.cpp:108-116).
struct PoissonBuffer {
  Dims D;
  int nz_hat;
  size_t stridex, stridey, stridez;
  std::vector<Real> data;
  FFTPlan px, py, pz;
  void init(const Dims& D_) {
    D = D_;
    nz_hat = D.nz / 2 + 1;
    stridez = 1; stridey = 2 * (size_t)nz_hat; stridex = (size_t)D.ny * 2 * nz_hat;
    data.assign((size_t)D.nx * stridex, 0.0);
    px.init(D.nx); py.init(D.ny); pz.init(D.nz);
  }
  size_t dest(int x, int y, int z) const { return stridex * x + stridey * y + stridez * z; }
  std::complex<Real>* cdata() { return reinterpret_cast<std::complex<Real>*>(data.data()); }
  size_t cidx(int kx, int ky, int kz) const { return ((size_t)kx * D.ny + ky) * nz_hat + kz; }

  // 3-D real-to-complex transform in place (FFTW r2c semantics; spectral
  // layout here is [kx][ky][kz] — FFTW_MPI_TRANSPOSED_OUT's [ky][kx][kz]
  // differs only in storage order, and _solve below indexes it accordingly).
  void r2c() {
    std::complex<Real>* c = cdata();
    #pragma omp parallel
    {
      std::vector<std::complex<Real>> line(std::max({D.nx, D.ny, D.nz}));
      #pragma omp for schedule(static) collapse(2)
      for (int x = 0; x < D.nx; ++x)
        for (int y = 0; y < D.ny; ++y) {
          Real* r = &data[dest(x, y, 0)];
          for (int z = 0; z < D.nz; ++z) line[z] = std::complex<Real>(r[z], 0.0);
          pz.exec(line.data(), -1);
          std::complex<Real>* o = c + cidx(x, y, 0);
          for (int k = 0; k < nz_hat; ++k) o[k] = line[k];
        }
      #pragma omp for schedule(static) collapse(2)
      for (int x = 0; x < D.nx; ++x)
        for (int k = 0; k < nz_hat; ++k) {
          for (int y = 0; y < D.ny; ++y) line[y] = c[cidx(x, y, k)];
          py.exec(line.data(), -1);
          for (int y = 0; y < D.ny; ++y) c[cidx(x, y, k)] = line[y];
        }
      #pragma omp for schedule(static) collapse(2)
      for (int y = 0; y < D.ny; ++y)
        for (int k = 0; k < nz_hat; ++k) {
          for (int x = 0; x < D.nx; ++x) line[x] = c[cidx(x, y, k)];
          px.exec(line.data(), -1);
          for (int x = 0; x < D.nx; ++x) c[cidx(x, y, k)] = line[x];
        }
    }
  }
  // 3-D complex-to-real transform in place (FFTW c2r semantics, unnormalised).
  void c2r() {
    std::complex<Real>* c = cdata();
    #pragma omp parallel
    {
      std::vector<std::complex<Real>> line(std::max({D.nx, D.ny, D.nz}));
      #pragma omp for schedule(static) collapse(2)
      for (int y = 0; y < D.ny; ++y)
        for (int k = 0; k < nz_hat; ++k) {
          for (int x = 0; x < D.nx; ++x) line[x] = c[cidx(x, y, k)];
          px.exec(line.data(), +1);
          for (int x = 0; x < D.nx; ++x) c[cidx(x, y, k)] = line[x];
        }
      #pragma omp for schedule(static) collapse(2)
      for (int x = 0; x < D.nx; ++x)
        for (int k = 0; k < nz_hat; ++k) {
          for (int y = 0; y < D.ny; ++y) line[y] = c[cidx(x, y, k)];
          py.exec(line.data(), +1);
          for (int y = 0; y < D.ny; ++y) c[cidx(x, y, k)] = line[y];
        }
      #pragma omp for schedule(static) collapse(2)
      for (int x = 0; x < D.nx; ++x)
        for (int y = 0; y < D.ny; ++y) {
          std::complex<Real>* h = c + cidx(x, y, 0);
          for (int k = 0; k < nz_hat; ++k) line[k] = h[k];
          for (int k = nz_hat; k < D.nz; ++k) line[k] = std::conj(h[D.nz - k]);
          pz.exec(line.data(), +1);
          Real* r = &data[dest(x, y, 0)];
          for (int z = 0; z < D.nz; ++z) r[z] = line[z].real();
        }
    }
  }
};

// PoissonSolverPeriodic::_solve, grid-consistent branch
// (source/poisson/PoissonSolverPeriodic.cpp:15-61): spectral divide by the
// eigenvalue of the wide (2h) Laplacian, then zero the 8 undefined modes.
void poisson_solve(PoissonBuffer& B, Real h) {
  B.r2c();
  std::complex<Real>* in_out = B.cdata();
  const size_t gsize[3] = {(size_t)B.D.nx, (size_t)B.D.ny, (size_t)B.D.nz};
  const Real norm_factor = 4 / (gsize[0] * h * gsize[1] * gsize[2]);
  const long nKx = (long)gsize[0], nKy = (long)gsize[1], nKz = (long)gsize[2];
  const Real wFacX = 4 * M_PI / nKx, wFacY = 4 * M_PI / nKy, wFacZ = 4 * M_PI / nKz;
  const long nz_hat = B.nz_hat;
  #pragma omp parallel for schedule(static)
  for (long j = 0; j < nKy; ++j)
    for (long i = 0; i < nKx; ++i)
      for (long k = 0; k < nz_hat; ++k) {
        const size_t linidx = B.cidx((int)i, (int)j, (int)k);
        const Real D = std::cos(wFacX * i) + std::cos(wFacY * j) + std::cos(wFacZ * k);
        const Real solutionFactor = norm_factor / (2 * D - 6);
        in_out[linidx] = std::complex<Real>(in_out[linidx].real() * solutionFactor,
                                            in_out[linidx].imag() * solutionFactor);
      }
  const long lastI = nKx / 2, lastJ = nKy / 2, lastK = nKz / 2;
  const long Is[2] = {0, lastI}, Js[2] = {0, lastJ}, Ks[2] = {0, lastK};
  for (long a : Is) for (long b : Js) for (long c : Ks)
    in_out[B.cidx((int)a, (int)b, (int)c)] = std::complex<Real>(0, 0);
  B.c2r();
}

// ---------------------------------------------------------------------------
// Simulation state (the subset of SimulationData on the hot path,
// source/SimulationData.h:46-179) plus one optional sphere obstacle.
struct Sphere {
  Real radius = 0.1;
  double position[3] = {0.5, 0.5, 0.5};
  double transVel[3] = {0, 0, 0};
  double angVel[3] = {0, 0, 0};
  double centerOfMass[3] = {0, 0, 0};
  bool bForcedInSimFrame[3] = {false, false, false};
  bool bFixFrameOfRef[3] = {false, false, false};
  double lambda_factor = 1.0;        // source/obstacles/Obstacle.h:106
  double force[3] = {0, 0, 0}, torque[3] = {0, 0, 0};
  // rigid-body state of source/obstacles/Obstacle.h:94-130 for free dofs
  double transVel_imposed[3] = {0, 0, 0};
  bool bBlockRotation[3] = {false, false, false};
  double quaternion[4] = {1, 0, 0, 0};
  double mass = 0, J[6] = {0, 0, 0, 0, 0, 0};
  double transVel_computed[3] = {0, 0, 0}, angVel_computed[3] = {0, 0, 0};
  double penalM = 0, penalCM[3] = {0, 0, 0}, penalJ[6] = {0, 0, 0, 0, 0, 0};
  double penalLmom[3] = {0, 0, 0}, penalAmom[3] = {0, 0, 0};
  std::vector<char> touched;         // obstacle block present (ObstacleBlock* != nullptr)
  std::vector<Real> SDF, CHI;        // per cell, meaningful on touched blocks
  // surface points of ObstacleBlock::write (source/ObstacleBlock.h:157-166), in
  // block order and, per block, in the (iz, iy, ix) order they were found
  struct SurfacePoint {
    int gx, gy, gz;
    double dchidx, dchidy, dchidz, delta;
  };
  std::vector<int> surf_begin;       // per block: first surface point (nblocks + 1 entries)
  std::vector<SurfacePoint> surface;
};

}  // namespace

extern "C" {

typedef struct orc_config {
  int nx, ny, nz;           // cells per dimension (multiples of 16, powers of two)
  double maxextent;         // h = maxextent / max(nx, ny, nz)  (SimulationData.cpp:184-198)
  double nu, CFL, lambda, DLM;
  double uinf[3];
  int rampup;
  int implicit_penalization;
  int scheme;               // 0: reference central2 + Euler, 1: upwind3 + RK2 (Heun)
  int has_sphere;
  double sphere_radius, sphere_position[3], sphere_velocity[3];
  int sphere_forced[3], sphere_fix_frame[3];
} orc_config;

}  // extern "C"

namespace {

struct OState {
  orc_config cfg;
  Dims D;
  Real h;
  int step = 0;
  double time = 0, dt = 0, lambda = 0, uMax_measured = 0;
  double uinf[3];
  std::vector<Real> u, v, w, p, chi, tmpU, tmpV, tmpW;
  PoissonBuffer pois;
  bool has_sphere = false;
  Sphere sph;
  double rhs_sums[3] = {0, 0, 0};
  double corr = 0;
};

// findMaxU (source/operators/ProcessHelpers.h:74-99)
double find_max_u(const OState& S) {
  const Real uinf[3] = {S.uinf[0], S.uinf[1], S.uinf[2]};
  Real maxU = 0;
  const size_t n = S.D.n();
  #pragma omp parallel for schedule(static) reduction(max : maxU)
  for (size_t i = 0; i < n; ++i) {
    const Real advu = std::fabs(S.u[i] + uinf[0]);
    const Real advv = std::fabs(S.v[i] + uinf[1]);
    const Real advw = std::fabs(S.w[i] + uinf[2]);
    const Real maxUl = std::max({advu, advv, advw});
    maxU = std::max(maxU, maxUl);
  }
  return maxU;
}

// KernelAdvectDiffuse (source/operators/AdvectionDiffusion.cpp:111-144):
// central differences, explicit Euler; result into tmp.
void advect_diffuse_ref(OState& S, double dt) {
  const Dims D = S.D;
  const Real h = S.h;
  const Real mu = S.cfg.nu;
  const Real uInf[3] = {S.uinf[0], S.uinf[1], S.uinf[2]};
  for_each_block(D, [&](int bx, int by, int bz) {
    Lab Lu, Lv, Lw;
    Lu.load(S.u.data(), D, bx, by, bz, 1);
    Lv.load(S.v.data(), D, bx, by, bz, 1);
    Lw.load(S.w.data(), D, bx, by, bz, 1);
    const Real facA = -dt / (2 * h);
    const Real facD = (mu / h) * (dt / h);
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const Real Lu0 = Lu(ix, iy, iz), Lv0 = Lv(ix, iy, iz), Lw0 = Lw(ix, iy, iz);
      const Real dudx = Lu(ix+1,iy,iz) - Lu(ix-1,iy,iz), dvdx = Lv(ix+1,iy,iz) - Lv(ix-1,iy,iz), dwdx = Lw(ix+1,iy,iz) - Lw(ix-1,iy,iz);
      const Real dudy = Lu(ix,iy+1,iz) - Lu(ix,iy-1,iz), dvdy = Lv(ix,iy+1,iz) - Lv(ix,iy-1,iz), dwdy = Lw(ix,iy+1,iz) - Lw(ix,iy-1,iz);
      const Real dudz = Lu(ix,iy,iz+1) - Lu(ix,iy,iz-1), dvdz = Lv(ix,iy,iz+1) - Lv(ix,iy,iz-1), dwdz = Lw(ix,iy,iz+1) - Lw(ix,iy,iz-1);
      const Real uu = Lu0 + uInf[0], vv = Lv0 + uInf[1], ww = Lw0 + uInf[2];
      const Real duD = Lu(ix,iy+1,iz) + Lu(ix,iy-1,iz) + Lu(ix+1,iy,iz) + Lu(ix-1,iy,iz) + Lu(ix,iy,iz-1) + Lu(ix,iy,iz+1) - Lu0 * 6;
      const Real dvD = Lv(ix,iy+1,iz) + Lv(ix,iy-1,iz) + Lv(ix+1,iy,iz) + Lv(ix-1,iy,iz) + Lv(ix,iy,iz-1) + Lv(ix,iy,iz+1) - Lv0 * 6;
      const Real dwD = Lw(ix,iy+1,iz) + Lw(ix,iy-1,iz) + Lw(ix+1,iy,iz) + Lw(ix-1,iy,iz) + Lw(ix,iy,iz-1) + Lw(ix,iy,iz+1) - Lw0 * 6;
      const Real duA = uu * dudx + vv * dudy + ww * dudz;
      const Real dvA = uu * dvdx + vv * dvdy + ww * dvdz;
      const Real dwA = uu * dwdx + vv * dwdy + ww * dwdz;
      const size_t o = D.idx(bx * BS + ix, by * BS + iy, bz * BS + iz);
      S.tmpU[o] = Lu0 + facA * duA + facD * duD;
      S.tmpV[o] = Lv0 + facA * dvA + facD * dvD;
      S.tmpW[o] = Lw0 + facA * dwA + facD * dwD;
    }
  });
}

// Third-order upwind-biased first derivative times 6h, chosen by the sign of
// the advecting velocity a: for a > 0 (2f_{+1} + 3f_0 - 6f_{-1} + f_{-2}),
// otherwise (-f_{+2} + 6f_{+1} - 3f_0 - 2f_{-1}).
inline Real up3(Real a, Real fm2, Real fm1, Real f0, Real fp1, Real fp2) {
  return a > 0 ? (2 * fp1 + 3 * f0 - 6 * fm1 + fm2) : (-fp2 + 6 * fp1 - 3 * f0 - 2 * fm1);
}

// One explicit stage of upwind3 advection + central diffusion on the fields
// (a,b,c); output[i] = base + facA*adv + facD*lap, where the stage form is
//   stage 1: out = f + dt*A(f)
//   stage 2: out = 0.5*(f0 + (f1 + dt*A(f1)))
// This scheme is not in the reference snapshot (its KernelAdvectDiffuse is
// central2 + Euler); it follows the same block/lab structure.
void upwind3_stage(OState& S, double dt, const Real* a, const Real* b, const Real* c,
                   const Real* base_u, const Real* base_v, const Real* base_w,
                   Real* ou, Real* ov, Real* ow) {
  const Dims D = S.D;
  const Real h = S.h;
  const Real mu = S.cfg.nu;
  const Real uInf[3] = {S.uinf[0], S.uinf[1], S.uinf[2]};
  const Real facA = -dt / (6 * h);
  const Real facD = (mu / h) * (dt / h);
  for_each_block(D, [&](int bx, int by, int bz) {
    Lab L[3];
    L[0].load(a, D, bx, by, bz, 2);
    L[1].load(b, D, bx, by, bz, 2);
    L[2].load(c, D, bx, by, bz, 2);
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const Real uu = L[0](ix, iy, iz) + uInf[0];
      const Real vv = L[1](ix, iy, iz) + uInf[1];
      const Real ww = L[2](ix, iy, iz) + uInf[2];
      const size_t o = D.idx(bx * BS + ix, by * BS + iy, bz * BS + iz);
      Real* outs[3] = {ou, ov, ow};
      const Real* bases[3] = {base_u, base_v, base_w};
      for (int q = 0; q < 3; ++q) {
        const Lab& F = L[q];
        const Real f0 = F(ix, iy, iz);
        const Real dx = up3(uu, F(ix-2,iy,iz), F(ix-1,iy,iz), f0, F(ix+1,iy,iz), F(ix+2,iy,iz));
        const Real dy = up3(vv, F(ix,iy-2,iz), F(ix,iy-1,iz), f0, F(ix,iy+1,iz), F(ix,iy+2,iz));
        const Real dz = up3(ww, F(ix,iy,iz-2), F(ix,iy,iz-1), f0, F(ix,iy,iz+1), F(ix,iy,iz+2));
        const Real lap = F(ix,iy+1,iz) + F(ix,iy-1,iz) + F(ix+1,iy,iz) + F(ix-1,iy,iz) + F(ix,iy,iz-1) + F(ix,iy,iz+1) - f0 * 6;
        const Real adv = uu * dx + vv * dy + ww * dz;
        const Real t = f0 + facA * adv + facD * lap;
        outs[q][o] = bases[q] ? 0.5 * (bases[q][o] + t) : t;
      }
    }
  });
}

void advect_diffuse_upwind3_rk2(OState& S, double dt) {
  const size_t n = S.D.n();
  std::vector<Real> u1(n), v1(n), w1(n);
  upwind3_stage(S, dt, S.u.data(), S.v.data(), S.w.data(), nullptr, nullptr, nullptr,
                u1.data(), v1.data(), w1.data());
  upwind3_stage(S, dt, u1.data(), v1.data(), w1.data(), S.u.data(), S.v.data(), S.w.data(),
                S.tmpU.data(), S.tmpV.data(), S.tmpW.data());
}

// AdvectionDiffusion::operator() (source/operators/AdvectionDiffusion.cpp:402-428):
// kernel into tmp, then UpdateAndCorrectInflow_nonUniform copies tmp -> u
// (:315-397); its inflow correction is inactive on periodic boundaries.
void op_advection_diffusion(OState& S, double dt) {
  if (S.cfg.scheme == 1) advect_diffuse_upwind3_rk2(S, dt);
  else advect_diffuse_ref(S, dt);
  std::copy(S.tmpU.begin(), S.tmpU.end(), S.u.begin());
  std::copy(S.tmpV.begin(), S.tmpV.end(), S.v.begin());
  std::copy(S.tmpW.begin(), S.tmpW.end(), S.w.begin());
}

// Signed distance of a sphere (source/obstacles/Sphere.cpp:44-48), positive inside.
inline Real sphere_sdf(const Sphere& s, Real x, Real y, Real z) {
  const Real dx = x - s.position[0], dy = y - s.position[1], dz = z - s.position[2];
  return s.radius - std::sqrt(dx * dx + dy * dy + dz * dz);
}

// CreateObstacles for one sphere (source/operators/ObstaclesCreate.cpp:444-540):
// reset chi=0, tmpU=-1; SDF fill on touching blocks (source/obstacles/Sphere.cpp:19-49,
// source/obstacles/extra/ObstacleLibrary.h:45-62); characteristic function
// (ObstaclesCreate.cpp:51-136); grid centre of mass (:230-256).
void op_create_obstacles(OState& S) {
  if (!S.has_sphere) return;
  const Dims D = S.D;
  const Real h = S.h;
  Sphere& s = S.sph;
  std::fill(S.chi.begin(), S.chi.end(), 0.0);
  std::fill(S.tmpU.begin(), S.tmpU.end(), -1.0);
  // updateUinf (source/obstacles/ObstacleVector.h:60-76) and Obstacle::update
  // position advection (source/obstacles/Obstacle.cpp:314-321).
  for (int d = 0; d < 3; ++d) S.uinf[d] = s.bFixFrameOfRef[d] ? -s.transVel[d] : 0.0;
  for (int d = 0; d < 3; ++d) s.position[d] += S.dt * (s.transVel[d] + S.uinf[d]);
  {  // orientation (source/obstacles/Obstacle.cpp:323-346; the sphere's shape does not depend on it)
    const double* w = s.angVel;
    const double* Q = s.quaternion;
    const double dqdt[4] = {.5 * (-w[0] * Q[1] - w[1] * Q[2] - w[2] * Q[3]), .5 * (+w[0] * Q[0] + w[1] * Q[3] - w[2] * Q[2]),
                            .5 * (-w[0] * Q[3] + w[1] * Q[0] + w[2] * Q[1]), .5 * (+w[0] * Q[2] - w[1] * Q[1] + w[2] * Q[0])};
    const double DQ[4] = {dqdt[0] * S.dt, dqdt[1] * S.dt, dqdt[2] * S.dt, dqdt[3] * S.dt};
    const double DQn = std::sqrt(DQ[0] * DQ[0] + DQ[1] * DQ[1] + DQ[2] * DQ[2] + DQ[3] * DQ[3]);
    if (DQn > std::numeric_limits<double>::epsilon()) {
      const double tanF = std::tan(DQn) / DQn;
      const double Dq[4] = {Q[0] + tanF * DQ[0], Q[1] + tanF * DQ[1], Q[2] + tanF * DQ[2], Q[3] + tanF * DQ[3]};
      const double invD = 1 / std::sqrt(Dq[0] * Dq[0] + Dq[1] * Dq[1] + Dq[2] * Dq[2] + Dq[3] * Dq[3]);
      for (int k = 0; k < 4; ++k) s.quaternion[k] = Dq[k] * invD;
    }
  }
  const Real safety = (2 + SURFDH) * h;
  const Real box[3][2] = {
    {(Real)s.position[0] - (s.radius + safety), (Real)s.position[0] + (s.radius + safety)},
    {(Real)s.position[1] - (s.radius + safety), (Real)s.position[1] + (s.radius + safety)},
    {(Real)s.position[2] - (s.radius + safety), (Real)s.position[2] + (s.radius + safety)}};
  const int nb = D.nblocks();
  s.touched.assign(nb, 0);
  s.SDF.assign(D.n(), 0.0);
  s.CHI.assign(D.n(), 0.0);
  for (int b = 0; b < nb; ++b) {
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    const int bi[3] = {bx, by, bz};
    bool touch = true;
    for (int d = 0; d < 3; ++d) {
      const Real minp = (bi[d] * BS + 0.5) * h, maxp = (bi[d] * BS + BS - 1 + 0.5) * h;
      const Real lo = std::max(minp, box[d][0]), hi = std::min(maxp, box[d][1]);
      if (!(hi - lo > 0)) touch = false;
    }
    s.touched[b] = touch;
    if (!touch) continue;
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const int gx = bx * BS + ix, gy = by * BS + iy, gz = bz * BS + iz;
      const Real dist = sphere_sdf(s, (gx + 0.5) * h, (gy + 0.5) * h, (gz + 0.5) * h);
      const size_t o = D.idx(gx, gy, gz);
      s.SDF[o] = dist;
      S.tmpU[o] = std::max(dist, S.tmpU[o]);
    }
  }
  const Real inv2h = .5 / h, vol = h * h * h;
  double com[4] = {0, 0, 0, 0};
  s.surface.clear();
  s.surf_begin.assign(nb + 1, 0);
  for (int b = 0; b < nb; ++b) {
    if (!s.touched[b]) continue;
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    Lab L;
    L.load(S.tmpU.data(), D, bx, by, bz, 1);
    double m = 0, cx = 0, cy = 0, cz = 0;
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const int gx = bx * BS + ix, gy = by * BS + iy, gz = bz * BS + iz;
      const size_t o = D.idx(gx, gy, gz);
      const Real sdf = s.SDF[o];
      Real chi;
      if (sdf > +2 * h || sdf < -2 * h) {
        chi = sdf > 0 ? 1 : 0;
      } else {
        const Real distPx = L(ix+1,iy,iz), distMx = L(ix-1,iy,iz);
        const Real distPy = L(ix,iy+1,iz), distMy = L(ix,iy-1,iz);
        const Real distPz = L(ix,iy,iz+1), distMz = L(ix,iy,iz-1);
        const Real gradUX = inv2h * (distPx - distMx);
        const Real gradUY = inv2h * (distPy - distMy);
        const Real gradUZ = inv2h * (distPz - distMz);
        const Real gradUSq = gradUX * gradUX + gradUY * gradUY + gradUZ * gradUZ + EPS;
        const Real IplusX = distPx < 0 ? 0 : distPx, IminuX = distMx < 0 ? 0 : distMx;
        const Real IplusY = distPy < 0 ? 0 : distPy, IminuY = distMy < 0 ? 0 : distMy;
        const Real IplusZ = distPz < 0 ? 0 : distPz, IminuZ = distMz < 0 ? 0 : distMz;
        const Real gradIX = inv2h * (IplusX - IminuX);
        const Real gradIY = inv2h * (IplusY - IminuY);
        const Real gradIZ = inv2h * (IplusZ - IminuZ);
        const Real numH = gradIX * gradUX + gradIY * gradUY + gradIZ * gradUZ;
        chi = numH / gradUSq;
      }
      s.CHI[o] = chi;
      S.chi[o] = std::max(chi, S.chi[o]);
      const Real p[3] = {(gx + 0.5) * h, (gy + 0.5) * h, (gz + 0.5) * h};
      cx += chi * vol * p[0]; cy += chi * vol * p[1]; cz += chi * vol * p[2];
      m += chi * vol;
      // surface delta and normal with the SDF shifted outward by SURFDH cells
      // (ObstaclesCreate.cpp:106-131)
      const Real sdfs = sdf + h * SURFDH;
      if (sdfs > +2 * h || sdfs < -2 * h) continue;
      const Real dPx = L(ix+1,iy,iz) + h * SURFDH, dMx = L(ix-1,iy,iz) + h * SURFDH;
      const Real dPy = L(ix,iy+1,iz) + h * SURFDH, dMy = L(ix,iy-1,iz) + h * SURFDH;
      const Real dPz = L(ix,iy,iz+1) + h * SURFDH, dMz = L(ix,iy,iz-1) + h * SURFDH;
      const Real gUX = inv2h * (dPx - dMx), gUY = inv2h * (dPy - dMy), gUZ = inv2h * (dPz - dMz);
      const Real gUSq = gUX * gUX + gUY * gUY + gUZ * gUZ + EPS;
      auto Hs = [](Real d) -> Real { return std::fabs(d) < EPS ? 0.5 : (d < 0 ? 0 : 1); };
      const Real gHX = Hs(dPx) - Hs(dMx), gHY = Hs(dPy) - Hs(dMy), gHZ = Hs(dPz) - Hs(dMz);
      const Real numD = gHX * gUX + gHY * gUY + gHZ * gUZ;
      const Real Delta = .5 * h * h * numD / gUSq;  // h^3 * Delta
      if (Delta > EPS) s.surface.push_back({gx, gy, gz, -Delta * gUX, -Delta * gUY, -Delta * gUZ, Delta});
    }
    com[0] += m; com[1] += cx; com[2] += cy; com[3] += cz;
    s.surf_begin[b + 1] = (int)s.surface.size();
  }
  for (int b = 1; b <= nb; ++b) s.surf_begin[b] = std::max(s.surf_begin[b], s.surf_begin[b - 1]);
  s.centerOfMass[0] = com[1] / com[0];
  s.centerOfMass[1] = com[2] / com[0];
  s.centerOfMass[2] = com[3] / com[0];
}

// PressureRHS::operator() (source/operators/PressureRHS.cpp:273-346), uniform grid:
// KernelPressureRHS (:51-76), obstacle visitor (:78-112), correction factors
// (:331-334) and KernelFinalizePerimeters (:215-256).
void op_pressure_rhs(OState& S, double dt) {
  const Dims D = S.D;
  const Real h = S.h;
  PoissonBuffer& P = S.pois;
  std::fill(P.data.begin(), P.data.end(), 0.0);   // reset() (PoissonSolver.cpp:132-135)
  const Real fac = 0.5 * h * h / dt;
  for_each_block(D, [&](int bx, int by, int bz) {
    Lab Lu, Lv, Lw;
    Lu.load(S.u.data(), D, bx, by, bz, 1);
    Lv.load(S.v.data(), D, bx, by, bz, 1);
    Lw.load(S.w.data(), D, bx, by, bz, 1);
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix)
      P.data[P.dest(bx * BS + ix, by * BS + iy, bz * BS + iz)] =
          fac * (Lu(ix+1,iy,iz) - Lu(ix-1,iy,iz) + Lv(ix,iy+1,iz) - Lv(ix,iy-1,iz) + Lw(ix,iy,iz+1) - Lw(ix,iy,iz-1));
  });
  S.rhs_sums[0] = S.rhs_sums[1] = S.rhs_sums[2] = 0;
  S.corr = 0;
  if (!S.has_sphere) return;
  const Sphere& s = S.sph;
  std::vector<char> touchSurf(D.n(), 0);
  double sumRHS = 0, posRHS = 0, negRHS = 0;
  const int nb = D.nblocks();
  #pragma omp parallel for schedule(static) reduction(+ : sumRHS, posRHS, negRHS)
  for (int b = 0; b < nb; ++b) {
    if (!s.touched[b]) continue;
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    Lab Lc;
    Lc.load(S.chi.data(), D, bx, by, bz, 1);
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const int gx = bx * BS + ix, gy = by * BS + iy, gz = bz * BS + iz;
      const size_t o = D.idx(gx, gy, gz);
      if (Lc(ix, iy, iz) > s.CHI[o]) continue;
      const size_t idx = P.dest(gx, gy, gz);
      const Real dXx = Lc(ix+1,iy,iz) - Lc(ix-1,iy,iz);
      const Real dXy = Lc(ix,iy+1,iz) - Lc(ix,iy-1,iz);
      const Real dXz = Lc(ix,iy,iz+1) - Lc(ix,iy,iz-1);
      const bool bSurface = dXx * dXx + dXy * dXy + dXz * dXz > 0;
      if (bSurface) touchSurf[o] = 1;
      const Real srcBulk = -s.CHI[o] * P.data[idx];
      sumRHS += srcBulk;
      P.data[idx] += srcBulk;
      posRHS += bSurface * P.data[idx] * (P.data[idx] > 0);
      negRHS -= bSurface * P.data[idx] * (P.data[idx] < 0);
    }
  }
  const double corrDenom = sumRHS > 0 ? posRHS : negRHS;
  const double corr = sumRHS / std::max(corrDenom, (double)EPS);
  S.rhs_sums[0] = sumRHS; S.rhs_sums[1] = posRHS; S.rhs_sums[2] = negRHS;
  S.corr = corr;
  #pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    if (!s.touched[b]) continue;
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const int gx = bx * BS + ix, gy = by * BS + iy, gz = bz * BS + iz;
      if (!touchSurf[D.idx(gx, gy, gz)]) continue;
      Real& r = P.data[P.dest(gx, gy, gz)];
      if (r > 0 and corr > 0) r -= corr * r;
      else if (r < 0 and corr < 0) r += corr * r;
    }
  }
}

// PressureProjection::operator() (source/operators/PressureProjection.cpp:107-129):
// solve, _fftw2cub (source/poisson/PoissonSolver.cpp:116-130), KernelGradP (:38-50).
void op_pressure_projection(OState& S, double dt) {
  const Dims D = S.D;
  const Real h = S.h;
  poisson_solve(S.pois, h);
  #pragma omp parallel for schedule(static)
  for (int z = 0; z < D.nz; ++z)
    for (int y = 0; y < D.ny; ++y)
      for (int x = 0; x < D.nx; ++x) S.p[D.idx(x, y, z)] = S.pois.data[S.pois.dest(x, y, z)];
  const Real fac = -0.5 * dt / h;
  for_each_block(D, [&](int bx, int by, int bz) {
    Lab Lp;
    Lp.load(S.p.data(), D, bx, by, bz, 1);
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const size_t o = D.idx(bx * BS + ix, by * BS + iy, bz * BS + iz);
      S.u[o] += fac * (Lp(ix+1,iy,iz) - Lp(ix-1,iy,iz));
      S.v[o] += fac * (Lp(ix,iy+1,iz) - Lp(ix,iy-1,iz));
      S.w[o] += fac * (Lp(ix,iy,iz+1) - Lp(ix,iy,iz-1));
    }
  });
}

// Dense solve A x = b by LU with partial pivoting (the GSL LU routines that
// Obstacle::computeVelocities calls, source/obstacles/Obstacle.cpp:200-207).
void lu_solve6(double A[6][6], double b[6], double x[6]) {
  int perm[6] = {0, 1, 2, 3, 4, 5};
  for (int j = 0; j < 5; ++j) {
    int piv = j;
    double mx = std::fabs(A[j][j]);
    for (int i = j + 1; i < 6; ++i)
      if (std::fabs(A[i][j]) > mx) mx = std::fabs(A[i][j]), piv = i;
    if (piv != j) {
      for (int k = 0; k < 6; ++k) std::swap(A[j][k], A[piv][k]);
      std::swap(perm[j], perm[piv]);
    }
    if (A[j][j] == 0) continue;
    for (int i = j + 1; i < 6; ++i) {
      const double l = A[i][j] / A[j][j];
      A[i][j] = l;
      for (int k = j + 1; k < 6; ++k) A[i][k] -= l * A[j][k];
    }
  }
  double y[6];
  for (int i = 0; i < 6; ++i) y[i] = b[perm[i]];
  for (int i = 0; i < 6; ++i)
    for (int k = 0; k < i; ++k) y[i] -= A[i][k] * y[k];
  for (int i = 5; i >= 0; --i) {
    for (int k = i + 1; k < 6; ++k) y[i] -= A[i][k] * y[k];
    y[i] /= A[i][i];
  }
  for (int i = 0; i < 6; ++i) x[i] = y[i];
}

// UpdateObstacles (source/operators/ObstaclesUpdate.cpp:202-236):
// KernelIntegrateFluidMomenta (:24-134) over the obstacle blocks (cells with
// chi > 0, moments about the centre of mass; the sphere has no deformation
// velocity), KernelFinalizeObstacleVel (:136-200) and
// Obstacle::computeVelocities (source/obstacles/Obstacle.cpp:153-264): the
// 6x6 momentum balance, forced dofs and blocked rotations replaced by their
// imposed values; the computed velocities become the free dofs' velocities.
void op_update_obstacles(OState& S) {
  if (!S.has_sphere) return;
  const Dims D = S.D;
  const Real h = S.h;
  Sphere& s = S.sph;
  const bool implicitPen = S.cfg.implicit_penalization != 0;
  const double lambdt = S.lambda * S.dt;
  const double* CM = s.centerOfMass;
  const int nb = D.nblocks();
  double M[29] = {0};
  for (int b = 0; b < nb; ++b) {
    if (!s.touched[b]) continue;
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    double q[29] = {0};
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const int gx = bx * BS + ix, gy = by * BS + iy, gz = bz * BS + iz;
      const size_t o = D.idx(gx, gy, gz);
      if (s.CHI[o] <= 0) continue;
      double p[3] = {(gx + 0.5) * h, (gy + 0.5) * h, (gz + 0.5) * h};
      const double dv = h * h * h, X = s.CHI[o];
      p[0] -= CM[0]; p[1] -= CM[1]; p[2] -= CM[2];
      const double u = S.u[o], v = S.v[o], w = S.w[o];
      q[0] += X * dv;
      q[7] += X * dv * (p[1] * p[1] + p[2] * p[2]);
      q[8] += X * dv * (p[0] * p[0] + p[2] * p[2]);
      q[9] += X * dv * (p[0] * p[0] + p[1] * p[1]);
      q[10] -= X * dv * p[0] * p[1];
      q[11] -= X * dv * p[0] * p[2];
      q[12] -= X * dv * p[1] * p[2];
      q[1] += X * dv * u; q[2] += X * dv * v; q[3] += X * dv * w;
      q[4] += X * dv * (p[1] * w - p[2] * v);
      q[5] += X * dv * (p[2] * u - p[0] * w);
      q[6] += X * dv * (p[0] * v - p[1] * u);
      if (implicitPen) {
        const double penalFac = dv * lambdt * X / (1 + X * lambdt);
        q[13] += penalFac;
        q[14] += penalFac * p[0]; q[15] += penalFac * p[1]; q[16] += penalFac * p[2];
        q[17] += penalFac * (p[1] * p[1] + p[2] * p[2]);
        q[18] += penalFac * (p[0] * p[0] + p[2] * p[2]);
        q[19] += penalFac * (p[0] * p[0] + p[1] * p[1]);
        q[20] -= penalFac * p[0] * p[1];
        q[21] -= penalFac * p[0] * p[2];
        q[22] -= penalFac * p[1] * p[2];
        q[23] += penalFac * u; q[24] += penalFac * v; q[25] += penalFac * w;
        q[26] += penalFac * (p[1] * w - p[2] * v);
        q[27] += penalFac * (p[2] * u - p[0] * w);
        q[28] += penalFac * (p[0] * v - p[1] * u);
      }
    }
    for (int k = 0; k < 29; ++k) M[k] += q[k];
  }
  s.mass = M[0];
  for (int k = 0; k < 6; ++k) s.J[k] = M[7 + k];
  if (implicitPen) {
    s.penalM = M[13];
    for (int d = 0; d < 3; ++d) s.penalCM[d] = M[14 + d], s.penalLmom[d] = M[23 + d], s.penalAmom[d] = M[26 + d];
    for (int k = 0; k < 6; ++k) s.penalJ[k] = M[17 + k];
  } else {
    s.penalM = M[0];
    for (int d = 0; d < 3; ++d) s.penalCM[d] = 0, s.penalLmom[d] = M[1 + d], s.penalAmom[d] = M[4 + d];
    for (int k = 0; k < 6; ++k) s.penalJ[k] = M[7 + k];
  }
  const double pM = s.penalM, *pC = s.penalCM, *pJ = s.penalJ;
  double A[6][6] = {{pM, 0, 0, 0, +pC[2], -pC[1]},
                    {0, pM, 0, -pC[2], 0, +pC[0]},
                    {0, 0, pM, +pC[1], -pC[0], 0},
                    {0, -pC[2], +pC[1], pJ[0], pJ[3], pJ[4]},
                    {+pC[2], 0, -pC[0], pJ[3], pJ[1], pJ[5]},
                    {-pC[1], +pC[0], 0, pJ[4], pJ[5], pJ[2]}};
  double b[6] = {s.penalLmom[0], s.penalLmom[1], s.penalLmom[2], s.penalAmom[0], s.penalAmom[1], s.penalAmom[2]};
  for (int d = 0; d < 3; ++d) {
    if (s.bForcedInSimFrame[d]) {
      for (int k = 0; k < 6; ++k)
        if (k != d) A[d][k] = 0;
      b[d] = pM * s.transVel_imposed[d];
    }
    if (s.bBlockRotation[d]) {
      for (int k = 0; k < 6; ++k)
        if (k != 3 + d) A[3 + d][k] = 0;
      b[3 + d] = 0;
    }
  }
  double x[6];
  lu_solve6(A, b, x);
  for (int d = 0; d < 3; ++d) s.transVel_computed[d] = x[d], s.angVel_computed[d] = x[3 + d];
  for (int d = 0; d < 3; ++d) s.force[d] = s.mass * (s.transVel_computed[d] - s.transVel[d]) / S.dt;
  const double dAv[3] = {(s.angVel_computed[0] - s.angVel[0]) / S.dt, (s.angVel_computed[1] - s.angVel[1]) / S.dt,
                         (s.angVel_computed[2] - s.angVel[2]) / S.dt};
  s.torque[0] = s.J[0] * dAv[0] + s.J[3] * dAv[1] + s.J[4] * dAv[2];
  s.torque[1] = s.J[3] * dAv[0] + s.J[1] * dAv[1] + s.J[5] * dAv[2];
  s.torque[2] = s.J[4] * dAv[0] + s.J[5] * dAv[1] + s.J[2] * dAv[2];
  for (int d = 0; d < 3; ++d) {
    s.transVel[d] = s.bForcedInSimFrame[d] ? s.transVel_imposed[d] : s.transVel_computed[d];
    s.angVel[d] = s.bBlockRotation[d] ? 0.0 : s.angVel_computed[d];
  }
}

// Penalization::operator() (source/operators/Penalization.cpp:129-156):
// KernelPenalization<implicit> (:40-98) + KernelFinalizePenalizationForce (:101-123).
void op_penalization(OState& S, double dt) {
  if (!S.has_sphere) return;
  const Dims D = S.D;
  const Real h = S.h;
  Sphere& s = S.sph;
  const bool implicitPen = S.cfg.implicit_penalization != 0;
  const double lambda = S.lambda, invdt = 1.0 / dt;
  const std::array<double, 3> CM = {s.centerOfMass[0], s.centerOfMass[1], s.centerOfMass[2]};
  const std::array<double, 3> vel = {s.transVel[0], s.transVel[1], s.transVel[2]};
  const std::array<double, 3> omega = {s.angVel[0], s.angVel[1], s.angVel[2]};
  const Real dv = std::pow(h, 3);
  const double lambdaFac = s.lambda_factor * (implicitPen ? lambda : invdt);
  double M[6] = {0, 0, 0, 0, 0, 0};
  const int nb = D.nblocks();
  #pragma omp parallel for schedule(static) reduction(+ : M[:6])
  for (int b = 0; b < nb; ++b) {
    if (!s.touched[b]) continue;
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    double FX = 0, FY = 0, FZ = 0, TX = 0, TY = 0, TZ = 0;
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const int gx = bx * BS + ix, gy = by * BS + iy, gz = bz * BS + iz;
      const size_t o = D.idx(gx, gy, gz);
      if (S.chi[o] > s.CHI[o]) continue;
      if (s.CHI[o] <= 0) continue;
      double p[3] = {(gx + 0.5) * h, (gy + 0.5) * h, (gz + 0.5) * h};
      p[0] -= CM[0]; p[1] -= CM[1]; p[2] -= CM[2];
      const double X = s.CHI[o], U_TOT[3] = {
          vel[0] + omega[1] * p[2] - omega[2] * p[1],
          vel[1] + omega[2] * p[0] - omega[0] * p[2],
          vel[2] + omega[0] * p[1] - omega[1] * p[0]};
      const Real penalFac = implicitPen ? X * lambdaFac / (1 + lambdaFac * dt * X) : X * lambdaFac;
      const Real FPX = penalFac * (U_TOT[0] - S.u[o]);
      const Real FPY = penalFac * (U_TOT[1] - S.v[o]);
      const Real FPZ = penalFac * (U_TOT[2] - S.w[o]);
      S.u[o] = S.u[o] + dt * FPX;
      S.v[o] = S.v[o] + dt * FPY;
      S.w[o] = S.w[o] + dt * FPZ;
      FX += dv * FPX; FY += dv * FPY; FZ += dv * FPZ;
      TX += dv * (p[1] * FPZ - p[2] * FPY);
      TY += dv * (p[2] * FPX - p[0] * FPZ);
      TZ += dv * (p[0] * FPY - p[1] * FPX);
    }
    M[0] += FX; M[1] += FY; M[2] += FZ; M[3] += TX; M[4] += TY; M[5] += TZ;
  }
  for (int d = 0; d < 3; ++d) { s.force[d] = M[d]; s.torque[d] = M[3 + d]; }
}

// ---------------------------------------------------------------------------
// Tangent-linear model of the step (test infrastructure: the FP64 directional
// derivative that GPU adjoints are checked against). The advecting-velocity
// signs of the upwind stencil are frozen at the base state; the projection is
// linear and applied to the tangent as is; penalization scales by (1 - dt pf).

// Tangent of one explicit stage S(f) = f + facA sum_d a_d D_d(f) + facD Lap f
// at base f = (a,b,c) along g = (ga,gb,gc); stage-2 form when base_g given:
// out = 0.5 (base_g + S'(f) g).
void stage_tangent(OState& S, double dt, const Real* a, const Real* b, const Real* c, const Real* ga,
                   const Real* gb, const Real* gc, const Real* bg_u, const Real* bg_v, const Real* bg_w, Real* ou,
                   Real* ov, Real* ow) {
  const Dims D = S.D;
  const Real h = S.h;
  const Real mu = S.cfg.nu;
  const bool up = S.cfg.scheme == 1;
  const Real uInf[3] = {S.uinf[0], S.uinf[1], S.uinf[2]};
  const Real facA = up ? -dt / (6 * h) : -dt / (2 * h);
  const Real facD = (mu / h) * (dt / h);
  const int g = up ? 2 : 1;
  for_each_block(D, [&](int bx, int by, int bz) {
    Lab F[3], T[3];
    F[0].load(a, D, bx, by, bz, g); F[1].load(b, D, bx, by, bz, g); F[2].load(c, D, bx, by, bz, g);
    T[0].load(ga, D, bx, by, bz, g); T[1].load(gb, D, bx, by, bz, g); T[2].load(gc, D, bx, by, bz, g);
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const Real adv[3] = {F[0](ix, iy, iz) + uInf[0], F[1](ix, iy, iz) + uInf[1], F[2](ix, iy, iz) + uInf[2]};
      const Real dadv[3] = {T[0](ix, iy, iz), T[1](ix, iy, iz), T[2](ix, iy, iz)};
      const size_t o = D.idx(bx * BS + ix, by * BS + iy, bz * BS + iz);
      Real* outs[3] = {ou, ov, ow};
      const Real* bgs[3] = {bg_u, bg_v, bg_w};
      // mean0: the derivative of a up3(a; f) with respect to a, which at a = 0
      // (a kink: one-sided derivatives up3(+; f) and up3(-; f)) is taken as
      // the mean of the two, (f-2 - 8 f-1 + 8 f+1 - f+2) / 2, what central
      // differences see
      auto deriv = [&](const Lab& L, int d, Real av, bool mean0) -> Real {
        const int ex = d == 0, ey = d == 1, ez = d == 2;
        const Real fm2 = up ? L(ix - 2 * ex, iy - 2 * ey, iz - 2 * ez) : 0, fp2 = up ? L(ix + 2 * ex, iy + 2 * ey, iz + 2 * ez) : 0;
        const Real fm1 = L(ix - ex, iy - ey, iz - ez), fp1 = L(ix + ex, iy + ey, iz + ez), f0 = L(ix, iy, iz);
        if (up && mean0 && av == 0) return 0.5 * (fm2 - 8 * fm1 + 8 * fp1 - fp2);
        return up ? up3(av, fm2, fm1, f0, fp1, fp2) : fp1 - fm1;
      };
      for (int q = 0; q < 3; ++q) {
        Real dA = 0;
        for (int d = 0; d < 3; ++d) dA += dadv[d] * deriv(F[q], d, adv[d], true) + adv[d] * deriv(T[q], d, adv[d], false);
        const Lab& G = T[q];
        const Real lap = G(ix,iy+1,iz) + G(ix,iy-1,iz) + G(ix+1,iy,iz) + G(ix-1,iy,iz) + G(ix,iy,iz-1) + G(ix,iy,iz+1) - G(ix,iy,iz) * 6;
        const Real t = G(ix, iy, iz) + facA * dA + facD * lap;
        outs[q][o] = bgs[q] ? 0.5 * (bgs[q][o] + t) : t;
      }
    }
  });
}

// P applied to the fields (a,b,c) in place: the pipeline's RHS, periodic
// Poisson solve and gradient correction on them (dt cancels in P; the
// pressure field of the state is overwritten).
void project_fields(OState& S, std::vector<Real>& a, std::vector<Real>& b, std::vector<Real>& c, double dt) {
  std::swap(S.u, a);
  std::swap(S.v, b);
  std::swap(S.w, c);
  op_pressure_rhs(S, dt);
  op_pressure_projection(S, dt);
  std::swap(S.u, a);
  std::swap(S.v, b);
  std::swap(S.w, c);
}

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_num_threads(int n) { if (n > 0) omp_set_num_threads(n); }

void* orc_create(const orc_config* cfg) {
  if (!cfg) return nullptr;
  const int N[3] = {cfg->nx, cfg->ny, cfg->nz};
  for (int d = 0; d < 3; ++d)
    if (N[d] < BS || N[d] % BS || !is_pow2(N[d])) return nullptr;
  OState* S = new OState();
  S->cfg = *cfg;
  S->D = Dims{cfg->nx, cfg->ny, cfg->nz};
  const double maxbpd = std::max({(double)N[0], (double)N[1], (double)N[2]});
  S->h = cfg->maxextent / maxbpd;
  S->lambda = cfg->lambda;
  for (int d = 0; d < 3; ++d) S->uinf[d] = cfg->uinf[d];
  const size_t n = S->D.n();
  for (auto* f : {&S->u, &S->v, &S->w, &S->p, &S->chi, &S->tmpU, &S->tmpV, &S->tmpW}) f->assign(n, 0.0);
  S->pois.init(S->D);
  if (cfg->has_sphere) {
    S->has_sphere = true;
    Sphere& s = S->sph;
    s.radius = cfg->sphere_radius;
    for (int d = 0; d < 3; ++d) {
      s.position[d] = cfg->sphere_position[d];
      s.bForcedInSimFrame[d] = cfg->sphere_forced[d] != 0;
      s.bFixFrameOfRef[d] = cfg->sphere_fix_frame[d] != 0;
      if (s.bForcedInSimFrame[d]) s.transVel_imposed[d] = s.transVel[d] = cfg->sphere_velocity[d];
    }
    // any forced dof blocks rotation (source/obstacles/Obstacle.cpp:131-137)
    const bool anyForced = s.bForcedInSimFrame[0] || s.bForcedInSimFrame[1] || s.bForcedInSimFrame[2];
    for (int d = 0; d < 3; ++d) s.bBlockRotation[d] = anyForced;
    // Initial CreateObstacles call with dt = 0 (source/Simulation.cpp:399-400).
    S->dt = 0;
    op_create_obstacles(*S);
  }
  return S;
}

void orc_destroy(void* h) { delete static_cast<OState*>(h); }

double orc_h(void* h) { return static_cast<OState*>(h)->h; }

void orc_set_velocity(void* hdl, const double* u, const double* v, const double* w) {
  OState* S = static_cast<OState*>(hdl);
  const size_t n = S->D.n();
  std::copy(u, u + n, S->u.begin());
  std::copy(v, v + n, S->v.begin());
  std::copy(w, w + n, S->w.begin());
}

// which: 0 u, 1 v, 2 w, 3 p, 4 chi, 5 tmpU, 6 tmpV, 7 tmpW, 8 rhs (buffer, unpadded view)
void orc_get_field(void* hdl, int which, double* out) {
  OState* S = static_cast<OState*>(hdl);
  const Dims D = S->D;
  const std::vector<Real>* f = nullptr;
  switch (which) {
    case 0: f = &S->u; break; case 1: f = &S->v; break; case 2: f = &S->w; break;
    case 3: f = &S->p; break; case 4: f = &S->chi; break;
    case 5: f = &S->tmpU; break; case 6: f = &S->tmpV; break; case 7: f = &S->tmpW; break;
    case 8:
      for (int z = 0; z < D.nz; ++z) for (int y = 0; y < D.ny; ++y) for (int x = 0; x < D.nx; ++x)
        out[D.idx(x, y, z)] = S->pois.data[S->pois.dest(x, y, z)];
      return;
    default: return;
  }
  std::copy(f->begin(), f->end(), out);
}

// Simulation::calcMaxTimestep (source/Simulation.cpp:403-424).
double orc_calc_max_timestep(void* hdl) {
  OState* S = static_cast<OState*>(hdl);
  const double hMin = S->h, CFL = S->cfg.CFL;
  S->uMax_measured = find_max_u(*S);
  const double dtDif = hMin * hMin / S->cfg.nu;
  const double dtAdv = hMin / (S->uMax_measured + 1e-8);
  S->dt = CFL * std::min(dtDif, dtAdv);
  if (S->step < S->cfg.rampup) {
    const double x = (S->step + 1.0) / S->cfg.rampup;
    const double rampCFL = std::exp(std::log(1e-3) * (1 - x) + std::log(CFL) * x);
    S->dt = rampCFL * std::min(dtDif, dtAdv);
  }
  if (S->cfg.DLM > 0) S->lambda = S->cfg.DLM / S->dt;
  return S->dt;
}

double orc_max_u(void* hdl) { return find_max_u(*static_cast<OState*>(hdl)); }

// ComputeForces (source/operators/FluidSolidForces.cpp:17-158, 200-222) on the
// surface points of the last CreateObstacles: per block, the stress integrands
// of KernelComputeForces at each point (lab of u, v, w, p with a one-cell
// halo), summed per block in ObstacleBlock::sumQoI order
// (source/ObstacleBlock.h:81-93), then over blocks; then the derived powers of
// Obstacle::computeForces (source/obstacles/Obstacle.cpp:266-295) and the
// grid mass. out[27]; all zero without an obstacle.
void orc_compute_forces(void* hdl, double* out) {
  OState* S = static_cast<OState*>(hdl);
  for (int k = 0; k < 27; ++k) out[k] = 0;
  if (!S->has_sphere) return;
  const Dims D = S->D;
  const Sphere& s = S->sph;
  const Real h = S->h, _1oH = S->cfg.nu / h;
  const double* CM = s.centerOfMass;
  const double* uTrans = s.transVel;
  const double* omega = s.angVel;
  double velUnit[3] = {0., 0., 0.};
  const double vel_norm = std::sqrt(uTrans[0] * uTrans[0] + uTrans[1] * uTrans[1] + uTrans[2] * uTrans[2]);
  if (vel_norm > 1e-9)
    for (int d = 0; d < 3; ++d) velUnit[d] = uTrans[d] / vel_norm;
  const int nb = D.nblocks();
  std::vector<double> sum(22, 0.0);
  for (int b = 0; b < nb; ++b) {
    if (!s.touched[b] || s.surf_begin[b + 1] == s.surf_begin[b]) continue;
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    Lab LU, LV, LW;
    LU.load(S->u.data(), D, bx, by, bz, 1);
    LV.load(S->v.data(), D, bx, by, bz, 1);
    LW.load(S->w.data(), D, bx, by, bz, 1);
    double q[22] = {0};
    for (int i = s.surf_begin[b]; i < s.surf_begin[b + 1]; ++i) {
      const Sphere::SurfacePoint& sp = s.surface[i];
      const int ix = sp.gx - bx * BS, iy = sp.gy - by * BS, iz = sp.gz - bz * BS;
      const Real p[3] = {(sp.gx + 0.5) * h, (sp.gy + 0.5) * h, (sp.gz + 0.5) * h};
      const double D11 = _1oH * (LU(ix+1,iy,iz) - LU(ix-1,iy,iz));
      const double D22 = _1oH * (LV(ix,iy+1,iz) - LV(ix,iy-1,iz));
      const double D33 = _1oH * (LW(ix,iy,iz+1) - LW(ix,iy,iz-1));
      const double D12 = .5 * _1oH * (LU(ix,iy+1,iz) - LU(ix,iy-1,iz) + LV(ix+1,iy,iz) - LV(ix-1,iy,iz));
      const double D13 = .5 * _1oH * (LU(ix,iy,iz+1) - LU(ix,iy,iz-1) + LW(ix+1,iy,iz) - LW(ix-1,iy,iz));
      const double D23 = .5 * _1oH * (LW(ix,iy+1,iz) - LW(ix,iy-1,iz) + LV(ix,iy,iz+1) - LV(ix,iy,iz-1));
      const double P = S->p[D.idx(sp.gx, sp.gy, sp.gz)];
      const double normX = sp.dchidx, normY = sp.dchidy, normZ = sp.dchidz;
      const double fXV = D11 * normX + D12 * normY + D13 * normZ;
      const double fYV = D12 * normX + D22 * normY + D23 * normZ;
      const double fZV = D13 * normX + D23 * normY + D33 * normZ;
      const double fXP = -P * normX, fYP = -P * normY, fZP = -P * normZ;
      const double fXT = fXV + fXP, fYT = fYV + fYP, fZT = fZV + fZP;
      const double vX = LU(ix,iy,iz), vY = LV(ix,iy,iz), vZ = LW(ix,iy,iz);
      q[12] += normY * vZ - normZ * vY;
      q[13] += normZ * vX - normX * vZ;
      q[14] += normX * vY - normY * vX;
      q[0] += fXT; q[1] += fYT; q[2] += fZT;
      q[6] += fXV; q[7] += fYV; q[8] += fZV;
      q[3] += fXP; q[4] += fYP; q[5] += fZP;
      q[9] += (p[1] - CM[1]) * fZT - (p[2] - CM[2]) * fYT;
      q[10] += (p[2] - CM[2]) * fXT - (p[0] - CM[0]) * fZT;
      q[11] += (p[0] - CM[0]) * fYT - (p[1] - CM[1]) * fXT;
      const double forcePar = fXT * velUnit[0] + fYT * velUnit[1] + fZT * velUnit[2];
      q[16] += .5 * (forcePar + std::fabs(forcePar));
      q[15] -= .5 * (forcePar - std::fabs(forcePar));
      const double powOut = fXT * vX + fYT * vY + fZT * vZ;
      const double powDef = 0;  // the sphere has no deformation velocity
      q[17] += powOut; q[18] += std::min(0.0, powOut);
      q[19] += powDef; q[20] += std::min(0.0, powDef);
      const double rVec[3] = {p[0] - CM[0], p[1] - CM[1], p[2] - CM[2]};
      const double uSolid[3] = {uTrans[0] + omega[1] * rVec[2] - rVec[1] * omega[2],
                                uTrans[1] + omega[2] * rVec[0] - rVec[2] * omega[0],
                                uTrans[2] + omega[0] * rVec[1] - rVec[0] * omega[1]};
      q[21] += fXT * uSolid[0] + fYT * uSolid[1] + fZT * uSolid[2];
    }
    for (int k = 0; k < 22; ++k) sum[k] += q[k];
  }
  for (int k = 0; k < 22; ++k) out[k] = sum[k];
  const double drag = sum[15], thrust = sum[16], defPower = sum[19], defPowerBnd = sum[20];
  out[22] = thrust * vel_norm;
  out[23] = drag * vel_norm;
  out[24] = out[22] / (out[22] - std::min(defPower, 0.0) + EPS);
  out[25] = out[22] / (out[22] - defPowerBnd + EPS);
  double mass = 0;
  const Real vol = h * h * h;
  for (int b = 0; b < nb; ++b) {
    if (!s.touched[b]) continue;
    const int bx = b % D.bpd(0), by = (b / D.bpd(0)) % D.bpd(1), bz = b / (D.bpd(0) * D.bpd(1));
    double m = 0;
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) m += s.CHI[D.idx(bx * BS + ix, by * BS + iy, bz * BS + iz)] * vol;
    mass += m;
  }
  out[26] = mass;
}

// Pipeline operators by reference name (source/Simulation.cpp:307-401).
int orc_operator(void* hdl, const char* name, double dt) {
  OState* S = static_cast<OState*>(hdl);
  S->dt = dt;
  const std::string n(name);
  if (n == "CreateObstacles") op_create_obstacles(*S);
  else if (n == "AdvectionDiffusion") op_advection_diffusion(*S, dt);
  else if (n == "PressureRHS") op_pressure_rhs(*S, dt);
  else if (n == "PressureProjection") op_pressure_projection(*S, dt);
  else if (n == "UpdateObstacles") op_update_obstacles(*S);
  else if (n == "Penalization") op_penalization(*S, dt);
  else if (n == "ComputeForces") {}  // diagnostics only (orc_compute_forces): no state change
  else if (n == "ComputeDissipation") {}  // diagnostics only (orc_dissipation): no state change
  else return 1;
  return 0;
}

// Simulation::timestep (source/Simulation.cpp:593-623) over the hot-path pipeline.
void orc_timestep(void* hdl, double dt) {
  OState* S = static_cast<OState*>(hdl);
  S->dt = dt;
  if (S->has_sphere) op_create_obstacles(*S);
  op_advection_diffusion(*S, dt);
  op_pressure_rhs(*S, dt);
  op_pressure_projection(*S, dt);
  op_update_obstacles(*S);
  op_penalization(*S, dt);
  S->step++;
  S->time += dt;
}

// Runs nsteps of calcMaxTimestep + timestep; writes the dt sequence if dts != NULL.
// If fixed_dts != NULL, replays that dt sequence instead of calcMaxTimestep.
void orc_run(void* hdl, int nsteps, const double* fixed_dts, double* dts) {
  OState* S = static_cast<OState*>(hdl);
  for (int i = 0; i < nsteps; ++i) {
    double dt;
    if (fixed_dts) {
      orc_calc_max_timestep(hdl);
      dt = fixed_dts[i];
      S->dt = dt;
      if (S->cfg.DLM > 0) S->lambda = S->cfg.DLM / dt;
    } else {
      dt = orc_calc_max_timestep(hdl);
    }
    if (dts) dts[i] = dt;
    orc_timestep(hdl, dt);
  }
}

// stats: [0..2] force, [3..5] torque, [6] time, [7] step, [8..10] uinf,
// [11] dt, [12] lambda, [13..15] centre of mass, [16..18] rhs sums, [19] corr, [20] uMax
void orc_get_stats(void* hdl, double* out) {
  OState* S = static_cast<OState*>(hdl);
  for (int d = 0; d < 3; ++d) { out[d] = S->sph.force[d]; out[3 + d] = S->sph.torque[d]; }
  out[6] = S->time; out[7] = S->step;
  for (int d = 0; d < 3; ++d) out[8 + d] = S->uinf[d];
  out[11] = S->dt; out[12] = S->lambda;
  for (int d = 0; d < 3; ++d) out[13 + d] = S->sph.centerOfMass[d];
  for (int d = 0; d < 3; ++d) out[16 + d] = S->rhs_sums[d];
  out[19] = S->corr; out[20] = S->uMax_measured;
  for (int d = 0; d < 3; ++d) {
    out[21 + d] = S->sph.transVel[d];
    out[24 + d] = S->sph.angVel[d];
    out[27 + d] = S->sph.position[d];
  }
  for (int k = 0; k < 4; ++k) out[30 + k] = S->sph.quaternion[k];
}

// Stand-alone periodic Poisson solve of rhs (premultiplied by h^3, as the
// reference's PressureRHS leaves it) -> p, through the FFTW-layout buffer.
int orc_poisson_solve_field(int nx, int ny, int nz, double h, const double* rhs, double* p) {
  const int N[3] = {nx, ny, nz};
  for (int d = 0; d < 3; ++d) if (N[d] < 2 || !is_pow2(N[d])) return 1;
  PoissonBuffer B;
  Dims D{nx, ny, nz};
  B.init(D);
  for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x)
    B.data[B.dest(x, y, z)] = rhs[D.idx(x, y, z)];
  poisson_solve(B, h);
  for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x)
    p[D.idx(x, y, z)] = B.data[B.dest(x, y, z)];
  return 0;
}

// Restatement of tests/cubismup3d/TestBoundaries.cpp:19-52: through a periodic
// lab of halo g, out(cell) = lab(-dx,-dy,-dz) of f.
int orc_lab_shift(const double* f, double* out, int nx, int ny, int nz, int g, int dx, int dy, int dz) {
  Dims D{nx, ny, nz};
  if (nx % BS || ny % BS || nz % BS) return 1;
  if (std::abs(dx) > g || std::abs(dy) > g || std::abs(dz) > g) return 1;
  for_each_block(D, [&](int bx, int by, int bz) {
    Lab L;
    L.load(f, D, bx, by, bz, g);
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix)
      out[D.idx(bx * BS + ix, by * BS + iy, bz * BS + iz)] = L(ix - dx, iy - dy, iz - dz);
  });
  return 0;
}

// FP64 diagnostics: [0] kinetic energy sum h^3 |u|^2 / 2
// (source/operators/ComputeDissipation.cpp:47-116 pattern), [1] L2 norm of the
// central divergence (sum h^3 div^2)^(1/2), [2] max |div|.
void orc_diagnostics(void* hdl, double* out) {
  OState* S = static_cast<OState*>(hdl);
  const Dims D = S->D;
  const Real h = S->h, h3 = h * h * h, inv2h = 0.5 / h;
  double ke = 0, d2 = 0, dmax = 0;
  #pragma omp parallel for schedule(static) reduction(+ : ke, d2) reduction(max : dmax)
  for (int z = 0; z < D.nz; ++z)
    for (int y = 0; y < D.ny; ++y)
      for (int x = 0; x < D.nx; ++x) {
        const size_t o = D.idx(x, y, z);
        ke += 0.5 * h3 * (S->u[o] * S->u[o] + S->v[o] * S->v[o] + S->w[o] * S->w[o]);
        const double div = inv2h * (S->u[D.idx(wrap(x + 1, D.nx), y, z)] - S->u[D.idx(wrap(x - 1, D.nx), y, z)] +
                                    S->v[D.idx(x, wrap(y + 1, D.ny), z)] - S->v[D.idx(x, wrap(y - 1, D.ny), z)] +
                                    S->w[D.idx(x, y, wrap(z + 1, D.nz))] - S->w[D.idx(x, y, wrap(z - 1, D.nz))]);
        d2 += h3 * div * div;
        dmax = std::max(dmax, std::fabs(div));
      }
  out[0] = ke; out[1] = std::sqrt(d2); out[2] = dmax;
}

// ComputeDissipation (source/operators/ComputeDissipation.cpp:38-116, reduced
// as :119-160): per block, with a one-cell lab of u, v, w, p and the cell's
// chi, the 20 sums circulation[3], linImpulse[3], linMomentum[3],
// angImpulse[3], angMomentum[3], presPow, viscPow, helicity, kineticEn,
// enstrophy, in that order. Blocks are summed in block order.
void orc_dissipation(void* hdl, double* out) {
  OState* S = static_cast<OState*>(hdl);
  const Dims D = S->D;
  const Real h = S->h, nu = S->cfg.nu;
  const Real hCube = std::pow(h, 3), inv2h = .5 / h, invHh = 1 / (h * h);
  const Real center[3] = {D.nx * h / 2, D.ny * h / 2, D.nz * h / 2};
  const int nb = D.nblocks();
  std::vector<double> per((size_t)nb * 20, 0.0);
  for_each_block(D, [&](int bx, int by, int bz) {
    Lab Lu, Lv, Lw, Lp;
    Lu.load(S->u.data(), D, bx, by, bz, 1);
    Lv.load(S->v.data(), D, bx, by, bz, 1);
    Lw.load(S->w.data(), D, bx, by, bz, 1);
    Lp.load(S->p.data(), D, bx, by, bz, 1);
    double R[20] = {0};
    for (int iz = 0; iz < BS; ++iz)
    for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix) {
      const int gx = bx * BS + ix, gy = by * BS + iy, gz = bz * BS + iz;
      const Real X = S->has_sphere ? S->chi[D.idx(gx, gy, gz)] : 0.0;
      const Real PX = (gx + 0.5) * h - center[0], PY = (gy + 0.5) * h - center[1], PZ = (gz + 0.5) * h - center[2];
      const Real u = Lu(ix, iy, iz), v = Lv(ix, iy, iz), w = Lw(ix, iy, iz);
      const Real WX = inv2h * ((Lw(ix, iy + 1, iz) - Lw(ix, iy - 1, iz)) - (Lv(ix, iy, iz + 1) - Lv(ix, iy, iz - 1)));
      const Real WY = inv2h * ((Lu(ix, iy, iz + 1) - Lu(ix, iy, iz - 1)) - (Lw(ix + 1, iy, iz) - Lw(ix - 1, iy, iz)));
      const Real WZ = inv2h * ((Lv(ix + 1, iy, iz) - Lv(ix - 1, iy, iz)) - (Lu(ix, iy + 1, iz) - Lu(ix, iy - 1, iz)));
      const Real dPdx = inv2h * (Lp(ix + 1, iy, iz) - Lp(ix - 1, iy, iz));
      const Real dPdy = inv2h * (Lp(ix, iy + 1, iz) - Lp(ix, iy - 1, iz));
      const Real dPdz = inv2h * (Lp(ix, iy, iz + 1) - Lp(ix, iy, iz - 1));
      R[15] -= (1 - X) * hCube * (dPdx * u + dPdy * v + dPdz * w);
      const Real lapU = invHh * (Lu(ix + 1, iy, iz) + Lu(ix - 1, iy, iz) + Lu(ix, iy + 1, iz) + Lu(ix, iy - 1, iz) +
                                 Lu(ix, iy, iz + 1) + Lu(ix, iy, iz - 1) - 6 * u);
      const Real lapV = invHh * (Lv(ix + 1, iy, iz) + Lv(ix - 1, iy, iz) + Lv(ix, iy + 1, iz) + Lv(ix, iy - 1, iz) +
                                 Lv(ix, iy, iz + 1) + Lv(ix, iy, iz - 1) - 6 * v);
      const Real lapW = invHh * (Lw(ix + 1, iy, iz) + Lw(ix - 1, iy, iz) + Lw(ix, iy + 1, iz) + Lw(ix, iy - 1, iz) +
                                 Lw(ix, iy, iz + 1) + Lw(ix, iy, iz - 1) - 6 * w);
      const Real V1 = lapU * u + lapV * v + lapW * w;
      const Real D11 = inv2h * (Lu(ix + 1, iy, iz) - Lu(ix - 1, iy, iz));
      const Real D22 = inv2h * (Lv(ix, iy + 1, iz) - Lv(ix, iy - 1, iz));
      const Real D33 = inv2h * (Lw(ix, iy, iz + 1) - Lw(ix, iy, iz - 1));
      const Real D12 = inv2h * (Lu(ix, iy + 1, iz) - Lu(ix, iy - 1, iz) + Lv(ix + 1, iy, iz) - Lv(ix - 1, iy, iz)) / 2;
      const Real D13 = inv2h * (Lu(ix, iy, iz + 1) - Lu(ix, iy, iz - 1) + Lw(ix + 1, iy, iz) - Lw(ix - 1, iy, iz)) / 2;
      const Real D23 = inv2h * (Lw(ix, iy + 1, iz) - Lw(ix, iy - 1, iz) + Lv(ix, iy, iz + 1) - Lv(ix, iy, iz - 1)) / 2;
      const Real V2 = D11 * D11 + D22 * D22 + D33 * D33 + 2 * (D12 * D12 + D13 * D13 + D23 * D23);
      R[16] += (1 - X) * hCube * nu * (V1 + 2 * V2);
      R[0] += hCube * WX;
      R[1] += hCube * WY;
      R[2] += hCube * WZ;
      R[3] += hCube / 2 * (PY * WZ - PZ * WY);
      R[4] += hCube / 2 * (PZ * WX - PX * WZ);
      R[5] += hCube / 2 * (PX * WY - PY * WX);
      R[6] += hCube * u;
      R[7] += hCube * v;
      R[8] += hCube * w;
      R[9] += hCube / 3 * (PX * (PY * WY + PZ * WZ) - WX * (PY * PY + PZ * PZ));
      R[10] += hCube / 3 * (PY * (PX * WX + PZ * WZ) - WY * (PX * PX + PZ * PZ));
      R[11] += hCube / 3 * (PZ * (PX * WX + PY * WY) - WZ * (PX * PX + PY * PY));
      R[12] += hCube * (PY * w - PZ * v);
      R[13] += hCube * (PZ * u - PX * w);
      R[14] += hCube * (PX * v - PY * u);
      R[17] += hCube * (WX * u + WY * v + WZ * w);
      R[18] += hCube * (u * u + v * v + w * w) / 2;
      R[19] += std::sqrt(WX * WX + WY * WY + WZ * WZ);
    }
    const int b = bx + D.bpd(0) * (by + D.bpd(1) * bz);
    for (int k = 0; k < 20; ++k) per[(size_t)b * 20 + k] = R[k];
  });
  for (int k = 0; k < 20; ++k) out[k] = 0.0;
  for (int b = 0; b < nb; ++b)
    for (int k = 0; k < 20; ++k) out[k] += per[(size_t)b * 20 + k];
}

// Tangent-linear rollout (no obstacle): advances the state nsteps with the
// given dt sequence and the tangent (du, dv, dw) along with it, in place.
// Returns 1 if the state has an obstacle (not supported), else 0.
int orc_tangent_run(void* hdl, int nsteps, const double* dts, double* du, double* dv, double* dw) {
  OState* S = static_cast<OState*>(hdl);
  if (S->has_sphere) return 1;
  const size_t n = S->D.n();
  std::vector<Real> tu(du, du + n), tv(dv, dv + n), tw(dw, dw + n);
  std::vector<Real> u1(n), v1(n), w1(n), t1u(n), t1v(n), t1w(n);
  for (int s = 0; s < nsteps; ++s) {
    const double dt = dts[s];
    S->dt = dt;
    if (S->cfg.scheme == 1) {
      // u1 = S(u), du1 = S'(u) du
      upwind3_stage(*S, dt, S->u.data(), S->v.data(), S->w.data(), nullptr, nullptr, nullptr, u1.data(), v1.data(),
                    w1.data());
      stage_tangent(*S, dt, S->u.data(), S->v.data(), S->w.data(), tu.data(), tv.data(), tw.data(), nullptr, nullptr,
                    nullptr, t1u.data(), t1v.data(), t1w.data());
      // u* = 0.5 (u + S(u1)), du* = 0.5 (du + S'(u1) du1)
      std::vector<Real> su(n), sv(n), sw(n);
      stage_tangent(*S, dt, u1.data(), v1.data(), w1.data(), t1u.data(), t1v.data(), t1w.data(), tu.data(), tv.data(),
                    tw.data(), su.data(), sv.data(), sw.data());
      tu.swap(su);
      tv.swap(sv);
      tw.swap(sw);
      upwind3_stage(*S, dt, u1.data(), v1.data(), w1.data(), S->u.data(), S->v.data(), S->w.data(), S->tmpU.data(),
                    S->tmpV.data(), S->tmpW.data());
    } else {
      std::vector<Real> su(n), sv(n), sw(n);
      stage_tangent(*S, dt, S->u.data(), S->v.data(), S->w.data(), tu.data(), tv.data(), tw.data(), nullptr, nullptr,
                    nullptr, su.data(), sv.data(), sw.data());
      tu.swap(su);
      tv.swap(sv);
      tw.swap(sw);
      advect_diffuse_ref(*S, dt);
    }
    std::copy(S->tmpU.begin(), S->tmpU.end(), S->u.begin());
    std::copy(S->tmpV.begin(), S->tmpV.end(), S->v.begin());
    std::copy(S->tmpW.begin(), S->tmpW.end(), S->w.begin());
    op_pressure_rhs(*S, dt);
    op_pressure_projection(*S, dt);
    project_fields(*S, tu, tv, tw, dt);
    S->step++;
    S->time += dt;
  }
  std::copy(tu.begin(), tu.end(), du);
  std::copy(tv.begin(), tv.end(), dv);
  std::copy(tw.begin(), tw.end(), dw);
  return 0;
}

}  // extern "C"
