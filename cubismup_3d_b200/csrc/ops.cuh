// Per-cell operators run by k_stencil_stream, and the small kernels that
// work only on the obstacle's active box (sphere chi, RHS obstacle terms,
// penalization). Every operator cites the reference kernel it replaces.
#pragma once

#include "common.cuh"
#include "stencil.cuh"

namespace cup {

__device__ __forceinline__ size_t gidx(int x, int y, int z, int nx, int ny) {
  return ((size_t)z * ny + y) * nx + x;
}

// periodic wrap of an index at most one period outside [0, n)
__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Time step argument: host value, or a device scalar when chaining steps on
// the GPU without a host round trip (the CFL dt is computed on the device).
struct DtArg {
  double host;
  const double* dev;
  __device__ __forceinline__ double get() const { return dev ? *dev : host; }
};

// ---------------------------------------------------------------------------
// KernelAdvectDiffuse (source/operators/AdvectionDiffusion.cpp:111-144):
// central 2nd-order advection + 7-point diffusion, explicit Euler, into tmp.
template <typename T>
struct OpAdvectDiffuseRef {
  T *ou, *ov, *ow;
  DtArg dt;
  double h, nu;
  double uinf[3];
  int nx, ny;
  template <class C>
  __device__ __forceinline__ void cell(const C& c, int x, int y, int gy, int gz, double* acc) const {
    const double dtv = dt.get();
    const T facA = (T)(-dtv / (2 * h));
    const T facD = (T)((nu / h) * (dtv / h));
    const T Lu = c.v(0, x, y, 0, 0, 0), Lv = c.v(1, x, y, 0, 0, 0), Lw = c.v(2, x, y, 0, 0, 0);
    const T uE = c.v(0, x, y, 1, 0, 0), uW = c.v(0, x, y, -1, 0, 0), uN = c.v(0, x, y, 0, 1, 0),
            uS = c.v(0, x, y, 0, -1, 0), uB = c.v(0, x, y, 0, 0, 1), uF = c.v(0, x, y, 0, 0, -1);
    const T vE = c.v(1, x, y, 1, 0, 0), vW = c.v(1, x, y, -1, 0, 0), vN = c.v(1, x, y, 0, 1, 0),
            vS = c.v(1, x, y, 0, -1, 0), vB = c.v(1, x, y, 0, 0, 1), vF = c.v(1, x, y, 0, 0, -1);
    const T wE = c.v(2, x, y, 1, 0, 0), wW = c.v(2, x, y, -1, 0, 0), wN = c.v(2, x, y, 0, 1, 0),
            wS = c.v(2, x, y, 0, -1, 0), wB = c.v(2, x, y, 0, 0, 1), wF = c.v(2, x, y, 0, 0, -1);
    const T dudx = uE - uW, dvdx = vE - vW, dwdx = wE - wW;
    const T dudy = uN - uS, dvdy = vN - vS, dwdy = wN - wS;
    const T dudz = uB - uF, dvdz = vB - vF, dwdz = wB - wF;
    const T u = Lu + (T)uinf[0], v = Lv + (T)uinf[1], w = Lw + (T)uinf[2];
    const T duD = uN + uS + uE + uW + uF + uB - Lu * 6;
    const T dvD = vN + vS + vE + vW + vF + vB - Lv * 6;
    const T dwD = wN + wS + wE + wW + wF + wB - Lw * 6;
    const T duA = u * dudx + v * dudy + w * dudz;
    const T dvA = u * dvdx + v * dvdy + w * dvdz;
    const T dwA = u * dwdx + v * dwdy + w * dwdz;
    const size_t o = gidx(x, gy, gz, nx, ny);
    ou[o] = Lu + facA * duA + facD * duD;
    ov[o] = Lv + facA * dvA + facD * dvD;
    ow[o] = Lw + facA * dwA + facD * dwD;
  }
  __device__ void finish(double*, double*) const {}
};

// Third-order upwind-biased first derivative (times 6h) by the sign of the
// advecting velocity a: a > 0 -> (2f+1 + 3f0 - 6f-1 + f-2), else
// (-f+2 + 6f+1 - 3f0 - 2f-1). Not in the reference snapshot, whose
// KernelAdvectDiffuse is central + Euler; this is the scheme named for the
// B200 build, restated identically in the oracle.
template <typename T>
__device__ __forceinline__ T up3(T a, T fm2, T fm1, T f0, T fp1, T fp2) {
  return a > (T)0 ? ((T)2 * fp1 + (T)3 * f0 - (T)6 * fm1 + fm2) : (-fp2 + (T)6 * fp1 - (T)3 * f0 - (T)2 * fm1);
}

// One RK2 (Heun) stage of upwind3 advection + 7-point diffusion:
//   stage 1: out = f + dt A(f)
//   stage 2: out = 0.5 (f^n + (f1 + dt A(f1)))      (f^n read point-wise)
template <typename T, bool STAGE2>
struct OpUpwind3Stage {
  const T *bu, *bv, *bw;  // f^n, stage 2 only
  T *ou, *ov, *ow;
  DtArg dt;
  double h, nu;
  double uinf[3];
  int nx, ny;
  template <class C>
  __device__ __forceinline__ void cell(const C& c, int x, int y, int gy, int gz, double* acc) const {
    const double dtv = dt.get();
    const T facA = (T)(-dtv / (6 * h));
    const T facD = (T)((nu / h) * (dtv / h));
    const T uu = c.v(0, x, y, 0, 0, 0) + (T)uinf[0];
    const T vv = c.v(1, x, y, 0, 0, 0) + (T)uinf[1];
    const T ww = c.v(2, x, y, 0, 0, 0) + (T)uinf[2];
    const size_t o = gidx(x, gy, gz, nx, ny);
    T* outs[3] = {ou, ov, ow};
    const T* bases[3] = {bu, bv, bw};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const T f0 = c.v(q, x, y, 0, 0, 0);
      const T fxm2 = c.v(q, x, y, -2, 0, 0), fxm1 = c.v(q, x, y, -1, 0, 0), fxp1 = c.v(q, x, y, 1, 0, 0),
              fxp2 = c.v(q, x, y, 2, 0, 0);
      const T fym2 = c.v(q, x, y, 0, -2, 0), fym1 = c.v(q, x, y, 0, -1, 0), fyp1 = c.v(q, x, y, 0, 1, 0),
              fyp2 = c.v(q, x, y, 0, 2, 0);
      const T fzm2 = c.v(q, x, y, 0, 0, -2), fzm1 = c.v(q, x, y, 0, 0, -1), fzp1 = c.v(q, x, y, 0, 0, 1),
              fzp2 = c.v(q, x, y, 0, 0, 2);
      const T dx = up3(uu, fxm2, fxm1, f0, fxp1, fxp2);
      const T dy = up3(vv, fym2, fym1, f0, fyp1, fyp2);
      const T dz = up3(ww, fzm2, fzm1, f0, fzp1, fzp2);
      const T lap = fyp1 + fym1 + fxp1 + fxm1 + fzm1 + fzp1 - f0 * 6;
      const T adv = uu * dx + vv * dy + ww * dz;
      const T t = f0 + facA * adv + facD * lap;
      if (STAGE2) outs[q][o] = (T)0.5 * (bases[q][o] + t);
      else outs[q][o] = t;
    }
  }
  __device__ void finish(double*, double*) const {}
};

// KernelPressureRHS (source/operators/PressureRHS.cpp:51-76):
// rhs = (h^2 / 2dt) (du/dx + dv/dy + dw/dz) with central differences, i.e.
// h^3 div(u*) / dt; evaluated in FP64 whatever the storage type.
template <typename T>
struct OpPressureRHS {
  double* rhs;
  DtArg dt;
  double h;
  int nx, ny;
  template <class C>
  __device__ __forceinline__ void cell(const C& c, int x, int y, int gy, int gz, double* acc) const {
    const double fac = 0.5 * h * h / dt.get();
    const double uE = c.v(0, x, y, 1, 0, 0), uW = c.v(0, x, y, -1, 0, 0);
    const double vN = c.v(1, x, y, 0, 1, 0), vS = c.v(1, x, y, 0, -1, 0);
    const double wB = c.v(2, x, y, 0, 0, 1), wF = c.v(2, x, y, 0, 0, -1);
    rhs[gidx(x, gy, gz, nx, ny)] = fac * (uE - uW + vN - vS + wB - wF);
  }
  __device__ void finish(double*, double*) const {}
};

// FP64 defect of the Poisson equation, r = b - h^3 L_2h p, with L_2h the
// wide Laplacian sum_d (p(+2) - 2p + p(-2)) / (4h^2) that the spectral factor
// inverts (source/poisson/PoissonSolverPeriodic.cpp:19-37); written as FP32
// for the FP32 correction solve. Per-CTA FP64 partials: [0] sum r^2,
// [1] sum b^2, [2..9] sums of p and [10..17] sums of r over the 8 parity
// classes (x&1, y&1, z&1). The class sums give the components along the 8
// null modes of L_2h (mean and checkerboards), which the solve cannot change:
// they are removed from p (the mean-pressure fix) and left out of the
// convergence test.
struct OpResidual {
  const double* b;
  float* r;
  double* partials;     // [gridDim.x][18]
  const double* rmean;  // parity-class means of r from the first check (null parts), or nullptr
  double c;          // h / 4 = h^3 / (4 h^2)
  int nx, ny;
  template <class C>
  __device__ __forceinline__ void cell(const C& q, int x, int y, int gy, int gz, double* acc) const {
    const double p0 = q.v(0, x, y, 0, 0, 0);
    const double lx = q.v(0, x, y, 2, 0, 0) - 2 * p0 + q.v(0, x, y, -2, 0, 0);
    const double ly = q.v(0, x, y, 0, 2, 0) - 2 * p0 + q.v(0, x, y, 0, -2, 0);
    const double lz = q.v(0, x, y, 0, 0, 2) - 2 * p0 + q.v(0, x, y, 0, 0, -2);
    const size_t o = gidx(x, gy, gz, nx, ny);
    const double bb = b[o];
    const double res = bb - c * (lx + ly + lz);
    const int cls = (x & 1) | ((gy & 1) << 1) | ((gz & 1) << 2);
    // Null parts removed per cell, before the FP32 cast (their FP32 rounding
    // would otherwise feed the correction noise of their own size) and before
    // squaring (subtracting norms afterwards cancels catastrophically).
    const double rp = rmean ? res - rmean[cls] : res;
    r[o] = (float)rp;
    acc[0] += rp * rp;
    acc[1] += bb * bb;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      acc[2 + k] += (k == cls) ? p0 : 0.0;
      acc[10 + k] += (k == cls) ? res : 0.0;
    }
  }
  __device__ void finish(double* acc, double* scratch) const {
    double v[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) v[k] = acc[k];
    block_reduce<18, false>(v, scratch);
    if (threadIdx.x == 0)
      for (int k = 0; k < 18; ++k) partials[18 * blockIdx.x + k] = v[k];
  }
};

// ---- producers / consumers of the fused x pass (k_dht_rows) ---------------

// Rows of the pressure RHS computed from u* (KernelPressureRHS,
// source/operators/PressureRHS.cpp:51-76): fused into the first x pass so the
// RHS never goes to HBM.
template <typename T>
struct RowsRhs {
  const T *u, *v, *w;
  DtArg dt;
  double h;
  int nx, ny, nz;
  __device__ void fill(double* rows, int row0, int nr, int N) const {
    const double fac = 0.5 * h * h / dt.get();
    for (int i = threadIdx.x; i < nr * N; i += blockDim.x) {
      const int l = i / N, x = i - l * N;
      const int r = row0 + l, y = r % ny, z = r / ny;
      const double uE = u[gidx(wrapi(x + 1, nx), y, z, nx, ny)], uW = u[gidx(wrapi(x - 1, nx), y, z, nx, ny)];
      const double vN = v[gidx(x, wrapi(y + 1, ny), z, nx, ny)], vS = v[gidx(x, wrapi(y - 1, ny), z, nx, ny)];
      const double wB = w[gidx(x, y, wrapi(z + 1, nz), nx, ny)], wF = w[gidx(x, y, wrapi(z - 1, nz), nx, ny)];
      rows[i] = fac * (uE - uW + vN - vS + wB - wF);
    }
  }
};

// Active box of the obstacle: cells [lo, lo+n) per dimension (global indices,
// wrapped periodically). Outside it chi == 0 and the obstacle terms vanish.
struct Box {
  int lo[3], n[3];
  __device__ __forceinline__ bool contains(int x, int y, int z, int nx, int ny, int nz) const {
    int dx = x - lo[0]; dx += dx < 0 ? nx : 0;
    int dy = y - lo[1]; dy += dy < 0 ? ny : 0;
    int dz = z - lo[2]; dz += dz < 0 ? nz : 0;
    return dx < n[0] && dy < n[1] && dz < n[2];
  }
  __host__ __device__ __forceinline__ long long count() const { return (long long)n[0] * n[1] * n[2]; }
  // index of cell (x, y, z) in the box's [z][y][x] order, -1 outside
  __device__ __forceinline__ int index(int x, int y, int z, int nx, int ny, int nz) const {
    int dx = x - lo[0]; dx += dx < 0 ? nx : 0;
    int dy = y - lo[1]; dy += dy < 0 ? ny : 0;
    int dz = z - lo[2]; dz += dz < 0 ? nz : 0;
    return (dx < n[0] && dy < n[1] && dz < n[2]) ? dx + n[0] * (dy + n[1] * dz) : -1;
  }
};

// KernelGradP (source/operators/PressureProjection.cpp:38-50):
// u -= (dt/2h) (p(x+1) - p(x-1)) etc. Fused epilogue: per-CTA FP64 partials of
// max |u + uinf| (the next calcMaxTimestep, source/operators/ProcessHelpers.h:74-99)
// over cells outside the obstacle box (the penalization kernel covers the box)
// and the kinetic energy sum |u|^2/2 (ComputeDissipation.cpp:47-116 pattern).
template <typename T>
struct OpGradP {
  const T *su, *sv, *sw;  // u* (point-wise)
  T *ou, *ov, *ow;        // projected velocity
  double* partials;       // [gridDim.x][2]: max, ke
  DtArg dt;
  double h;
  double uinf[3];
  Box box;
  int has_box;
  int nx, ny, nz;
  template <class C>
  __device__ __forceinline__ void cell(const C& c, int x, int y, int gy, int gz, double* acc) const {
    const double fac = -0.5 * dt.get() / h;
    const double pE = c.v(0, x, y, 1, 0, 0), pW = c.v(0, x, y, -1, 0, 0);
    const double pN = c.v(0, x, y, 0, 1, 0), pS = c.v(0, x, y, 0, -1, 0);
    const double pB = c.v(0, x, y, 0, 0, 1), pF = c.v(0, x, y, 0, 0, -1);
    const size_t o = gidx(x, gy, gz, nx, ny);
    const double u = (double)su[o] + fac * (pE - pW);
    const double v = (double)sv[o] + fac * (pN - pS);
    const double w = (double)sw[o] + fac * (pB - pF);
    const T tu = (T)u, tv = (T)v, tw = (T)w;
    ou[o] = tu;
    ov[o] = tv;
    ow[o] = tw;
    if (!(has_box && box.contains(x, gy, gz, nx, ny, nz))) {
      const double m = fmax(fmax(fabs((double)tu + uinf[0]), fabs((double)tv + uinf[1])), fabs((double)tw + uinf[2]));
      acc[0] = fmax(acc[0], m);
    }
    acc[1] += 0.5 * ((double)tu * tu + (double)tv * tv + (double)tw * tw);
  }
  __device__ void finish(double* acc, double* scratch) const {
    double mx[1] = {acc[0]};
    double sm[1] = {acc[1]};
    block_reduce<1, true>(mx, scratch);
    block_reduce<1, false>(sm, scratch + 32);
    if (threadIdx.x == 0) {
      partials[2 * blockIdx.x + 0] = mx[0];
      partials[2 * blockIdx.x + 1] = sm[0];
    }
  }
};

// ---------------------------------------------------------------------------
// Obstacle-box kernels. Sphere parameters live in device memory so that the
// host can update them without relaunch changes.
struct SphereParams {
  double radius;
  double position[3];
  double transVel[3];
  double angVel[3];
  double centerOfMass[3];
  double lambda_factor;
  // rigid-body update of the free dofs (Obstacle::computeVelocities,
  // source/obstacles/Obstacle.cpp:153-264): forced translations keep
  // transVel_imposed; rotation is blocked when any translation is forced
  double transVel_imposed[3];
  int forced[3], block_rot[3];
  double mass, J[6];
  double transVel_computed[3], angVel_computed[3];
};

__device__ __forceinline__ double sphere_sdf(const SphereParams& s, double x, double y, double z) {
  const double dx = x - s.position[0], dy = y - s.position[1], dz = z - s.position[2];
  return s.radius - sqrt(dx * dx + dy * dy + dz * dz);
}


// KernelCharacteristicFunction (source/operators/ObstaclesCreate.cpp:51-136)
// with the sphere SDF of source/obstacles/Sphere.cpp:44-48 evaluated
// analytically at each (periodically wrapped) neighbour cell centre, plus the
// grid centre-of-mass partial sums (ObstaclesCreate.cpp:99-104, 230-256).
// One thread per box cell; writes chi (zero-initialised elsewhere).
template <typename T>
__global__ void k_sphere_chi(T* chi, const SphereParams* sp, Box box, int nx, int ny, int nz, double h,
                             double* partials /* [gridDim.x][4] */) {
  pdl_entry();
  __shared__ double scratch[4 * 32];
  const SphereParams s = *sp;
  double acc[4] = {0, 0, 0, 0};
  const long long n = box.count();
  const double EPS = 2.220446049250313080847e-16;  // std::numeric_limits<double>::epsilon()
  const double inv2h = .5 / h, vol = h * h * h;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(i % box.n[0]);
    const int by = (int)((i / box.n[0]) % box.n[1]);
    const int bz = (int)(i / ((long long)box.n[0] * box.n[1]));
    const int x = wrapi(box.lo[0] + bx, nx), y = wrapi(box.lo[1] + by, ny), z = wrapi(box.lo[2] + bz, nz);
    const double sdf = sphere_sdf(s, (x + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h);
    double X;
    if (sdf > +2 * h || sdf < -2 * h) {
      X = sdf > 0 ? 1 : 0;
    } else {
      const int xp = wrapi(x + 1, nx), xm = wrapi(x - 1, nx), yp = wrapi(y + 1, ny), ym = wrapi(y - 1, ny),
                zp = wrapi(z + 1, nz), zm = wrapi(z - 1, nz);
      const double distPx = sphere_sdf(s, (xp + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h);
      const double distMx = sphere_sdf(s, (xm + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h);
      const double distPy = sphere_sdf(s, (x + 0.5) * h, (yp + 0.5) * h, (z + 0.5) * h);
      const double distMy = sphere_sdf(s, (x + 0.5) * h, (ym + 0.5) * h, (z + 0.5) * h);
      const double distPz = sphere_sdf(s, (x + 0.5) * h, (y + 0.5) * h, (zp + 0.5) * h);
      const double distMz = sphere_sdf(s, (x + 0.5) * h, (y + 0.5) * h, (zm + 0.5) * h);
      const double gradUX = inv2h * (distPx - distMx);
      const double gradUY = inv2h * (distPy - distMy);
      const double gradUZ = inv2h * (distPz - distMz);
      const double gradUSq = gradUX * gradUX + gradUY * gradUY + gradUZ * gradUZ + EPS;
      const double IplusX = distPx < 0 ? 0 : distPx, IminuX = distMx < 0 ? 0 : distMx;
      const double IplusY = distPy < 0 ? 0 : distPy, IminuY = distMy < 0 ? 0 : distMy;
      const double IplusZ = distPz < 0 ? 0 : distPz, IminuZ = distMz < 0 ? 0 : distMz;
      const double gradIX = inv2h * (IplusX - IminuX);
      const double gradIY = inv2h * (IplusY - IminuY);
      const double gradIZ = inv2h * (IplusZ - IminuZ);
      const double numH = gradIX * gradUX + gradIY * gradUY + gradIZ * gradUZ;
      X = numH / gradUSq;
    }
    chi[gidx(x, y, z, nx, ny)] = (T)X;
    const double Xs = (double)(T)X;
    acc[0] += Xs * vol;
    acc[1] += Xs * vol * ((x + 0.5) * h);
    acc[2] += Xs * vol * ((y + 0.5) * h);
    acc[3] += Xs * vol * ((z + 0.5) * h);
  }
  block_reduce<4, false>(acc, scratch);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) partials[4 * blockIdx.x + k] = acc[k];
}

// Obstacle terms of KernelPressureRHS::visit (source/operators/PressureRHS.cpp:78-112)
// over the box: rhs -= chi rhs, surface tag where grad chi != 0 (central
// differences of chi), partial sums of the bulk source and of the positive /
// negative surface RHS.
template <typename T>
__global__ void k_rhs_obstacle(double* rhs, const T* chi, Box box, int nx, int ny, int nz,
                               double* partials /* [gridDim.x][3] */) {
  pdl_entry();
  __shared__ double scratch[3 * 32];
  double acc[3] = {0, 0, 0};
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const size_t o = gidx(x, y, z, nx, ny);
    const double X = chi[o];
    const double dXx = (double)chi[gidx(wrapi(x + 1, nx), y, z, nx, ny)] - (double)chi[gidx(wrapi(x - 1, nx), y, z, nx, ny)];
    const double dXy = (double)chi[gidx(x, wrapi(y + 1, ny), z, nx, ny)] - (double)chi[gidx(x, wrapi(y - 1, ny), z, nx, ny)];
    const double dXz = (double)chi[gidx(x, y, wrapi(z + 1, nz), nx, ny)] - (double)chi[gidx(x, y, wrapi(z - 1, nz), nx, ny)];
    const bool bSurface = dXx * dXx + dXy * dXy + dXz * dXz > 0;
    double r = rhs[o];
    const double srcBulk = -X * r;
    acc[0] += srcBulk;
    r += srcBulk;
    rhs[o] = r;
    acc[1] += bSurface * r * (r > 0);
    acc[2] -= bSurface * r * (r < 0);
  }
  block_reduce<3, false>(acc, scratch);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) partials[3 * blockIdx.x + k] = acc[k];
}

// KernelFinalizePerimeters (source/operators/PressureRHS.cpp:215-256) with the
// correction factor computed on the device (:331-334). BOXARR: rhs is an array
// over the box, and delta (holding b0, the RHS before its obstacle terms) is
// replaced by b2 - b0, the obstacle terms a pass that recomputes b0 from u*
// adds back on the box.
template <typename T, bool BOXARR = false>
__global__ void k_rhs_obstacle_correct(double* rhs, const T* chi, Box box, int nx, int ny, int nz,
                                       const double* corr_dev, double* delta = nullptr) {
  pdl_entry();
  const double corr = *corr_dev;
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const double dXx = (double)chi[gidx(wrapi(x + 1, nx), y, z, nx, ny)] - (double)chi[gidx(wrapi(x - 1, nx), y, z, nx, ny)];
    const double dXy = (double)chi[gidx(x, wrapi(y + 1, ny), z, nx, ny)] - (double)chi[gidx(x, wrapi(y - 1, ny), z, nx, ny)];
    const double dXz = (double)chi[gidx(x, y, wrapi(z + 1, nz), nx, ny)] - (double)chi[gidx(x, y, wrapi(z - 1, nz), nx, ny)];
    const size_t ro = BOXARR ? (size_t)i : gidx(x, y, z, nx, ny);
    double r = rhs[ro];
    if (dXx * dXx + dXy * dXy + dXz * dXz > 0) {
      if (r > 0 && corr > 0) r -= corr * r;
      else if (r < 0 && corr < 0) r += corr * r;
      if (!BOXARR) rhs[ro] = r;
    }
    if constexpr (BOXARR) delta[i] = r - delta[i];
  }
}

// b = KernelPressureRHS(u*) (source/operators/PressureRHS.cpp:51-76) as the
// FP32 defect-correction passes recompute it: the differences of the stored
// velocities and their sum in the storage type T, then one conversion to FP64
// and the scaling (one conversion per cell instead of six; T rounding of the
// differences is far below the storage rounding of u* itself). Every pass that
// recomputes b and the obstacle's box pass use these two functions, so b is
// the same bits wherever it is formed.
template <typename T>
__device__ __forceinline__ T div_xy(T uxp, T uxm, T vyp, T vym) {
  return (uxp - uxm) + (vyp - vym);
}
template <typename T>
__device__ __forceinline__ double div_b(double facB, T dxy, T wzp, T wzm) {
  return facB * (double)(dxy + (wzp - wzm));
}

// The first half of the RHS obstacle terms on the box, for passes that
// recompute b0 = KernelPressureRHS(u*) (source/operators/PressureRHS.cpp:51-76)
// themselves: b0 at each box cell (in the operation order of the z-queue
// passes' b from u*) into d, b1 = b0 - chi b0 into b (box [z][y][x] order), and
// the partial sums of k_rhs_obstacle (bulk source, positive / negative surface
// b1). k_rhs_obstacle_correct<T, true> then turns d into b2 - b0.
template <typename T>
__global__ void k_box_rhs_obstacle(const T* u, const T* v, const T* w, const T* chi, Box box, int nx, int ny, int nz,
                                   DtArg dt, double h, double* b, double* d, double* partials /* [gridDim.x][3] */) {
  pdl_entry();
  __shared__ double scratch[3 * 32];
  const double facB = 0.5 * h * h / dt.get();
  double acc[3] = {0, 0, 0};
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const size_t oxp = gidx(wrapi(x + 1, nx), y, z, nx, ny), oxm = gidx(wrapi(x - 1, nx), y, z, nx, ny);
    const size_t oyp = gidx(x, wrapi(y + 1, ny), z, nx, ny), oym = gidx(x, wrapi(y - 1, ny), z, nx, ny);
    const size_t ozp = gidx(x, y, wrapi(z + 1, nz), nx, ny), ozm = gidx(x, y, wrapi(z - 1, nz), nx, ny);
    const double b0 = div_b<T>(facB, div_xy<T>(u[oxp], u[oxm], v[oyp], v[oym]), w[ozp], w[ozm]);
    const double X = chi[gidx(x, y, z, nx, ny)];
    const double dXx = (double)chi[oxp] - (double)chi[oxm];
    const double dXy = (double)chi[oyp] - (double)chi[oym];
    const double dXz = (double)chi[ozp] - (double)chi[ozm];
    const bool bSurface = dXx * dXx + dXy * dXy + dXz * dXz > 0;
    const double srcBulk = -X * b0;
    acc[0] += srcBulk;
    const double r = b0 + srcBulk;
    acc[1] += bSurface * r * (r > 0);
    acc[2] -= bSurface * r * (r < 0);
    b[i] = r;
    d[i] = b0;
  }
  block_reduce<3, false>(acc, scratch);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) partials[3 * blockIdx.x + k] = acc[k];
}

// Surface forces of the sphere: the surface points of KernelCharacteristicFunction
// (source/operators/ObstaclesCreate.cpp:106-131: the SDF shifted outward by
// SURFDH cells, Heaviside differences of the neighbours, Delta = h^2/2 gradH .
// gradU / |gradU|^2 = h^3 delta, dchi = -Delta gradU) and, at each, the
// pressure and viscous stress integrands of KernelComputeForces
// (source/operators/FluidSolidForces.cpp:43-158) with the current u, v, w
// (central differences) and p; no rotation and no deformation velocity for the
// forced sphere. Per-CTA partials of the 22 quantities in ObstacleBlock::sumQoI
// order (source/ObstacleBlock.h:81-93): surface force, pressure force, viscous
// force, torque about the centre of mass, gamma, drag, thrust, Pout, PoutBnd,
// defPower, defPowerBnd, pLocom.
constexpr int kSurfQoI = 22;
template <typename T>
__global__ void k_surface_forces(const T* u, const T* v, const T* w, const double* p, const SphereParams* sp, Box box,
                                 int nx, int ny, int nz, double h, double nu, double* partials /* [gridDim.x][22] */) {
  pdl_entry();
  __shared__ double scratch[kSurfQoI * 32];
  const SphereParams s = *sp;
  double acc[kSurfQoI];
#pragma unroll
  for (int k = 0; k < kSurfQoI; ++k) acc[k] = 0.0;
  const double EPS = 2.220446049250313080847e-16;  // std::numeric_limits<double>::epsilon()
  const double inv2h = .5 / h, fac1 = .5 * h * h, shift = h * 1.0;  // SURFDH = 1
  const double _1oH = nu / h;
  const double* CM = s.centerOfMass;
  const double* uT = s.transVel;
  double velUnit[3] = {0., 0., 0.};
  const double vel_norm = sqrt(uT[0] * uT[0] + uT[1] * uT[1] + uT[2] * uT[2]);
  if (vel_norm > 1e-9) {
    velUnit[0] = uT[0] / vel_norm;
    velUnit[1] = uT[1] / vel_norm;
    velUnit[2] = uT[2] / vel_norm;
  }
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const double sdf = sphere_sdf(s, (x + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h) + shift;
    if (sdf > +2 * h || sdf < -2 * h) continue;
    const int xp = wrapi(x + 1, nx), xm = wrapi(x - 1, nx), yp = wrapi(y + 1, ny), ym = wrapi(y - 1, ny),
              zp = wrapi(z + 1, nz), zm = wrapi(z - 1, nz);
    const double distPx = sphere_sdf(s, (xp + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h) + shift;
    const double distMx = sphere_sdf(s, (xm + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h) + shift;
    const double distPy = sphere_sdf(s, (x + 0.5) * h, (yp + 0.5) * h, (z + 0.5) * h) + shift;
    const double distMy = sphere_sdf(s, (x + 0.5) * h, (ym + 0.5) * h, (z + 0.5) * h) + shift;
    const double distPz = sphere_sdf(s, (x + 0.5) * h, (y + 0.5) * h, (zp + 0.5) * h) + shift;
    const double distMz = sphere_sdf(s, (x + 0.5) * h, (y + 0.5) * h, (zm + 0.5) * h) + shift;
    const double gradUX = inv2h * (distPx - distMx);
    const double gradUY = inv2h * (distPy - distMy);
    const double gradUZ = inv2h * (distPz - distMz);
    const double gradUSq = gradUX * gradUX + gradUY * gradUY + gradUZ * gradUZ + EPS;
    auto H = [&](double d) { return fabs(d) < EPS ? 0.5 : (d < 0 ? 0.0 : 1.0); };
    const double gradHX = H(distPx) - H(distMx);
    const double gradHY = H(distPy) - H(distMy);
    const double gradHZ = H(distPz) - H(distMz);
    const double numD = gradHX * gradUX + gradHY * gradUY + gradHZ * gradUZ;
    const double Delta = fac1 * numD / gradUSq;
    if (!(Delta > EPS)) continue;
    const double normX = -Delta * gradUX, normY = -Delta * gradUY, normZ = -Delta * gradUZ;
    auto U = [&](const T* f, int a, int b, int c) { return (double)f[gidx(a, b, c, nx, ny)]; };
    const double D11 = _1oH * (U(u, xp, y, z) - U(u, xm, y, z));
    const double D22 = _1oH * (U(v, x, yp, z) - U(v, x, ym, z));
    const double D33 = _1oH * (U(w, x, y, zp) - U(w, x, y, zm));
    const double D12 = .5 * _1oH * (U(u, x, yp, z) - U(u, x, ym, z) + U(v, xp, y, z) - U(v, xm, y, z));
    const double D13 = .5 * _1oH * (U(u, x, y, zp) - U(u, x, y, zm) + U(w, xp, y, z) - U(w, xm, y, z));
    const double D23 = .5 * _1oH * (U(w, x, yp, z) - U(w, x, ym, z) + U(v, x, y, zp) - U(v, x, y, zm));
    const double P = p[gidx(x, y, z, nx, ny)];
    const double fXV = D11 * normX + D12 * normY + D13 * normZ;
    const double fYV = D12 * normX + D22 * normY + D23 * normZ;
    const double fZV = D13 * normX + D23 * normY + D33 * normZ;
    const double fXP = -P * normX, fYP = -P * normY, fZP = -P * normZ;
    const double fXT = fXV + fXP, fYT = fYV + fYP, fZT = fZV + fZP;
    const double px = (x + 0.5) * h, py = (y + 0.5) * h, pz = (z + 0.5) * h;
    const double vX = U(u, x, y, z), vY = U(v, x, y, z), vZ = U(w, x, y, z);
    acc[0] += fXT;
    acc[1] += fYT;
    acc[2] += fZT;
    acc[3] += fXP;
    acc[4] += fYP;
    acc[5] += fZP;
    acc[6] += fXV;
    acc[7] += fYV;
    acc[8] += fZV;
    acc[9] += (py - CM[1]) * fZT - (pz - CM[2]) * fYT;
    acc[10] += (pz - CM[2]) * fXT - (px - CM[0]) * fZT;
    acc[11] += (px - CM[0]) * fYT - (py - CM[1]) * fXT;
    acc[12] += normY * vZ - normZ * vY;
    acc[13] += normZ * vX - normX * vZ;
    acc[14] += normX * vY - normY * vX;
    const double forcePar = fXT * velUnit[0] + fYT * velUnit[1] + fZT * velUnit[2];
    acc[15] -= .5 * (forcePar - fabs(forcePar));  // drag
    acc[16] += .5 * (forcePar + fabs(forcePar));  // thrust
    const double powOut = fXT * vX + fYT * vY + fZT * vZ;
    acc[17] += powOut;
    acc[18] += fmin(0.0, powOut);
    // defPower, defPowerBnd: the sphere has no deformation velocity (acc[19], acc[20] stay 0)
    acc[21] += fXT * uT[0] + fYT * uT[1] + fZT * uT[2];  // pLocom with angVel = 0
  }
  block_reduce<kSurfQoI, false>(acc, scratch);
  if (threadIdx.x == 0)
    for (int k = 0; k < kSurfQoI; ++k) partials[kSurfQoI * blockIdx.x + k] = acc[k];
}

// KernelIntegrateFluidMomenta (source/operators/ObstaclesUpdate.cpp:24-134)
// over the box: for every cell with chi > 0, the volume, linear and angular
// momentum and inertia moments about the centre of mass and, for implicit
// penalization, the same weighted by dv lambda dt chi / (1 + chi lambda dt);
// the sphere has no deformation velocity. Per-CTA partials of the 29 sums in
// the order of KernelFinalizeObstacleVel (:142-160).
constexpr int kRigidQoI = 29;
template <typename T>
__global__ void k_integrate_momenta(const T* u, const T* v, const T* w, const T* chi, const SphereParams* sp, Box box,
                                    int nx, int ny, int nz, double h, DtArg dt, const double* lambda_dev,
                                    double lambda_host, int implicit_pen, double* partials /* [gridDim.x][29] */) {
  pdl_entry();
  __shared__ double scratch[kRigidQoI * 32];
  const SphereParams s = *sp;
  const double lambda = lambda_dev ? *lambda_dev : lambda_host;
  const double lambdt = lambda * dt.get();
  const double dv = h * h * h;
  double q[kRigidQoI];
#pragma unroll
  for (int k = 0; k < kRigidQoI; ++k) q[k] = 0.0;
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const size_t o = gidx(x, y, z, nx, ny);
    const double X = chi[o];
    if (X <= 0) continue;
    const double p0 = (x + 0.5) * h - s.centerOfMass[0], p1 = (y + 0.5) * h - s.centerOfMass[1],
                 p2 = (z + 0.5) * h - s.centerOfMass[2];
    const double uu = u[o], vv = v[o], ww = w[o];
    q[0] += X * dv;
    q[1] += X * dv * uu;
    q[2] += X * dv * vv;
    q[3] += X * dv * ww;
    q[4] += X * dv * (p1 * ww - p2 * vv);
    q[5] += X * dv * (p2 * uu - p0 * ww);
    q[6] += X * dv * (p0 * vv - p1 * uu);
    q[7] += X * dv * (p1 * p1 + p2 * p2);
    q[8] += X * dv * (p0 * p0 + p2 * p2);
    q[9] += X * dv * (p0 * p0 + p1 * p1);
    q[10] -= X * dv * p0 * p1;
    q[11] -= X * dv * p0 * p2;
    q[12] -= X * dv * p1 * p2;
    if (implicit_pen) {
      const double f = dv * lambdt * X / (1 + X * lambdt);
      q[13] += f;
      q[14] += f * p0;
      q[15] += f * p1;
      q[16] += f * p2;
      q[17] += f * (p1 * p1 + p2 * p2);
      q[18] += f * (p0 * p0 + p2 * p2);
      q[19] += f * (p0 * p0 + p1 * p1);
      q[20] -= f * p0 * p1;
      q[21] -= f * p0 * p2;
      q[22] -= f * p1 * p2;
      q[23] += f * uu;
      q[24] += f * vv;
      q[25] += f * ww;
      q[26] += f * (p1 * ww - p2 * vv);
      q[27] += f * (p2 * uu - p0 * ww);
      q[28] += f * (p0 * vv - p1 * uu);
    }
  }
  block_reduce<kRigidQoI, false>(q, scratch);
  if (threadIdx.x == 0)
    for (int k = 0; k < kRigidQoI; ++k) partials[kRigidQoI * blockIdx.x + k] = q[k];
}

// KernelPenalization<implicit> (source/operators/Penalization.cpp:40-98) over
// the box, FP64 force/torque partials (KernelFinalizePenalizationForce,
// :101-123) and the max |u + uinf| of every box cell after penalization.
template <typename T>
__global__ void k_penalize(T* u, T* v, T* w, const T* chi, const SphereParams* sp, Box box, int nx, int ny, int nz,
                           double h, DtArg dt, const double* lambda_dev, double lambda_host, int implicit_pen,
                           double uinf0, double uinf1, double uinf2, double* partials /* [gridDim.x][8] */) {
  pdl_entry();
  __shared__ double scratch[8 * 32];
  const SphereParams s = *sp;
  const double dtv = dt.get();
  const double lambda = lambda_dev ? *lambda_dev : lambda_host;
  const double lambdaFac = s.lambda_factor * (implicit_pen ? lambda : 1.0 / dtv);
  const double dv = h * h * h;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const size_t o = gidx(x, y, z, nx, ny);
    const double X = chi[o];
    double uu = u[o], vv = v[o], ww = w[o];
    if (X > 0) {
      double p[3] = {(x + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h};
      p[0] -= s.centerOfMass[0];
      p[1] -= s.centerOfMass[1];
      p[2] -= s.centerOfMass[2];
      const double U_TOT[3] = {s.transVel[0] + s.angVel[1] * p[2] - s.angVel[2] * p[1],
                               s.transVel[1] + s.angVel[2] * p[0] - s.angVel[0] * p[2],
                               s.transVel[2] + s.angVel[0] * p[1] - s.angVel[1] * p[0]};
      const double penalFac = implicit_pen ? X * lambdaFac / (1 + lambdaFac * dtv * X) : X * lambdaFac;
      const double FPX = penalFac * (U_TOT[0] - uu);
      const double FPY = penalFac * (U_TOT[1] - vv);
      const double FPZ = penalFac * (U_TOT[2] - ww);
      uu = uu + dtv * FPX;
      vv = vv + dtv * FPY;
      ww = ww + dtv * FPZ;
      u[o] = (T)uu;
      v[o] = (T)vv;
      w[o] = (T)ww;
      acc[0] += dv * FPX;
      acc[1] += dv * FPY;
      acc[2] += dv * FPZ;
      acc[3] += dv * (p[1] * FPZ - p[2] * FPY);
      acc[4] += dv * (p[2] * FPX - p[0] * FPZ);
      acc[5] += dv * (p[0] * FPY - p[1] * FPX);
    }
    const double tu = (T)uu, tv = (T)vv, tw = (T)ww;
    acc[6] = fmax(acc[6], fmax(fmax(fabs(tu + uinf0), fabs(tv + uinf1)), fabs(tw + uinf2)));
  }
  double sums[6] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5]};
  double mx[1] = {acc[6]};
  block_reduce<6, false>(sums, scratch);
  block_reduce<1, true>(mx, scratch + 6 * 32);
  if (threadIdx.x == 0) {
    for (int k = 0; k < 6; ++k) partials[8 * blockIdx.x + k] = sums[k];
    partials[8 * blockIdx.x + 6] = mx[0];
    partials[8 * blockIdx.x + 7] = 0;
  }
}

}  // namespace cup
