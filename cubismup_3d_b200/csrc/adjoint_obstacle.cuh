// Discrete adjoint of the obstacle terms of the step (no counterpart in the
// reference, which has no adjoint): the implicit / explicit Brinkman
// penalization (source/operators/Penalization.cpp:40-98) with its force
// (:101-123), and the obstacle terms of the pressure RHS
// (source/operators/PressureRHS.cpp:78-112, 215-256, 322-343).
//
// Forward, per step (box cells; chi = 0 outside the box):
//   b1 = (1 - chi) b0                      b0 = KernelPressureRHS(u*)
//   S = sum(-chi b0), corr = S / D          D = sum over the surface cells (grad chi != 0)
//                                           of b1 > 0 (S > 0) or of -b1 (b1 < 0, S < 0)
//   b2 = b1 (1 - sigma corr) on those cells (sigma = sign corr), b1 elsewhere
//   u** = u* - dt/(2h) grad_c L^+ b2
//   u' = u** + dt pf(chi) (U - u**)        pf = chi L / (1 + L dt chi) (implicit) or chi / dt
//   F = sum h^3 pf (U - u**)               (cells with chi > 0)
// The adjoint takes lambda = dJ/du' with J = <g, u_T> + sum_steps wF . F and
// returns dJ/du**, adds dJ/dchi and dJ/dU (the penalization target velocity U,
// the sphere's imposed translation, with uinf held fixed), and applies the
// transpose of the RHS map M: b0 -> b2. Linearised with the surface set and the
// sign of corr frozen (they only change where a surface b1 or S crosses zero;
// a surface cell whose b1 is exactly 0 takes the mean of the two sides).
// M db0 = m db0 - sigma b1_s dcorr, dcorr = c . db0, so
//   M^T q = m q - sigma (sum_s b1_s q_s) c,
//   m = (1 - chi)(1 - sigma corr [s]),  c_j = -chi_j / D - sigma S / D^2 (1 - chi_j) [s_j],
// and db2/dchi gives dJ/dchi_j = beta: -b0_j beta_j (1 - sigma corr [s_j]) - sigma (sum_s b1_s beta_s) e_j,
//   e_j = -b0_j / D + sigma S / D^2 b0_j [s_j],
// beta = dJ/db2. The chi gradient is the derivative from the chi >= 0 side
// (the forward leaves chi <= 0 cells unpenalized, so at chi = 0 it is the
// right derivative) and is reported on the box cells: outside the box the
// forward does not read chi.
#pragma once

#include "common.cuh"
#include "ops.cuh"

namespace cup {

struct ObstacleRhsState {
  double S, D, corr;  // sum of the bulk source, the corrected surface sum, the correction factor
  int sigma;          // sign of corr (0: no correction)
};

__device__ __forceinline__ ObstacleRhsState obstacle_rhs_state(const double* rhs_sums, double corr) {
  const double EPS = 2.220446049250313080847e-16;
  ObstacleRhsState s;
  s.S = rhs_sums[0];
  s.D = fmax(s.S > 0 ? rhs_sums[1] : rhs_sums[2], EPS);
  s.corr = corr;
  s.sigma = corr > 0 ? 1 : (corr < 0 ? -1 : 0);
  return s;
}

template <typename T>
__device__ __forceinline__ bool chi_surface(const T* chi, int x, int y, int z, int nx, int ny, int nz) {
  const double dXx = (double)chi[gidx(wrapi(x + 1, nx), y, z, nx, ny)] - (double)chi[gidx(wrapi(x - 1, nx), y, z, nx, ny)];
  const double dXy = (double)chi[gidx(x, wrapi(y + 1, ny), z, nx, ny)] - (double)chi[gidx(x, wrapi(y - 1, ny), z, nx, ny)];
  const double dXz = (double)chi[gidx(x, y, wrapi(z + 1, nz), nx, ny)] - (double)chi[gidx(x, y, wrapi(z - 1, nz), nx, ny)];
  return dXx * dXx + dXy * dXy + dXz * dXz > 0;
}

// Adjoint of the penalization and of the force term, over the box:
// lambda <- (1 - dt pf) lambda - h^3 pf wF (cells with chi > 0), g_chi +=
// pf'(chi) sum_c (U_c - u**_c)(dt lambda_c + h^3 wF_c), per-CTA partials of
// dJ/dU_c = sum pf (dt lambda_c + h^3 wF_c).
template <typename T>
__global__ void k_adj_penalize(T* lu, T* lv, T* lw, const T* su, const T* sv, const T* sw, const T* chi,
                               const SphereParams* sp, Box box, int nx, int ny, int nz, double h, double dt,
                               double Lfac, int implicit_pen, double wF0, double wF1, double wF2, double* g_chi,
                               double* partials /* [gridDim.x][3] */) {
  pdl_entry();
  __shared__ double scratch[3 * 32];
  const SphereParams s = *sp;
  const double dv = h * h * h;
  const double wF[3] = {wF0, wF1, wF2};
  double acc[3] = {0, 0, 0};
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const size_t o = gidx(x, y, z, nx, ny);
    const double X = chi[o];
    if (X < 0) continue;
    double p[3] = {(x + 0.5) * h - s.centerOfMass[0], (y + 0.5) * h - s.centerOfMass[1],
                   (z + 0.5) * h - s.centerOfMass[2]};
    const double U[3] = {s.transVel[0] + s.angVel[1] * p[2] - s.angVel[2] * p[1],
                         s.transVel[1] + s.angVel[2] * p[0] - s.angVel[0] * p[2],
                         s.transVel[2] + s.angVel[0] * p[1] - s.angVel[1] * p[0]};
    const double den = 1 + Lfac * dt * X;
    const double pf = implicit_pen ? X * Lfac / den : X * Lfac;
    const double dpf = implicit_pen ? Lfac / (den * den) : Lfac;
    const double us[3] = {(double)su[o], (double)sv[o], (double)sw[o]};
    T* lam[3] = {lu, lv, lw};
    double gx = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double l = lam[c][o];
      const double g = dt * l + dv * wF[c];
      gx += (U[c] - us[c]) * g;
      acc[c] += pf * g;
      if (X > 0) lam[c][o] = (T)((1 - dt * pf) * l - dv * pf * wF[c]);
    }
    g_chi[o] += dpf * gx;
  }
  block_reduce<3, false>(acc, scratch);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) partials[3 * blockIdx.x + k] = acc[k];
}

// Per-CTA partials of sum over the corrected surface cells of b1 q.
// rhs_sums: (S, positive, negative surface sums) and corr of the forward RHS.
template <typename T>
__global__ void k_adj_rhs_sum(const double* q, const double* b0, const T* chi, Box box, int nx, int ny, int nz,
                              const double* rhs_sums, const double* corr, double* partials /* [gridDim.x] */) {
  pdl_entry();
  __shared__ double scratch[32];
  const ObstacleRhsState rs = obstacle_rhs_state(rhs_sums, *corr);
  double acc[1] = {0};
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (rs.sigma == 0) break;
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const size_t o = gidx(x, y, z, nx, ny);
    const double b1 = b0[o] - (double)chi[o] * b0[o];
    if ((rs.sigma > 0 ? b1 > 0 : b1 < 0) && chi_surface(chi, x, y, z, nx, ny, nz)) acc[0] += b1 * q[o];
  }
  block_reduce<1, false>(acc, scratch);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

// q <- M^T q over the box and g_chi += kappa (db2/dchi)^T q, with kappa q =
// dJ/db2 and sq = the sum of k_adj_rhs_sum (read from *sq).
template <typename T>
__global__ void k_adj_rhs_apply(double* q, const double* b0, const T* chi, Box box, int nx, int ny, int nz,
                                const double* rhs_sums, const double* corr, const double* sq_dev, double kappa,
                                double* g_chi) {
  pdl_entry();
  const ObstacleRhsState rs = obstacle_rhs_state(rhs_sums, *corr);
  const double sq = rs.sigma != 0 ? *sq_dev : 0.0;
  const double invD = 1.0 / rs.D, SD2 = rs.S / (rs.D * rs.D);
  const long long n = box.count();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = wrapi(box.lo[0] + (int)(i % box.n[0]), nx);
    const int y = wrapi(box.lo[1] + (int)((i / box.n[0]) % box.n[1]), ny);
    const int z = wrapi(box.lo[2] + (int)(i / ((long long)box.n[0] * box.n[1])), nz);
    const size_t o = gidx(x, y, z, nx, ny);
    const double X = chi[o], B0 = b0[o], Q = q[o];
    const double b1 = B0 - X * B0;
    // weight of the cell in the corrected surface set: 1 inside it; 1/2 for
    // a surface b1 of exactly 0 that a perturbation can move (chi < 1), the
    // mean of the two sides' slopes, which central differences see (a flow
    // started from rest has such cells in its first step)
    double ws = 0.0;
    if (rs.sigma != 0 && chi_surface(chi, x, y, z, nx, ny, nz)) {
      if (rs.sigma > 0 ? b1 > 0 : b1 < 0) ws = 1.0;
      else if (b1 == 0 && X < 1) ws = 0.5;
    }
    const double fs = 1 - ws * rs.sigma * rs.corr;
    const double sig = (double)rs.sigma;
    const double cj = -X * invD - sig * SD2 * (1 - X) * ws;
    const double ej = -B0 * invD + sig * SD2 * B0 * ws;
    q[o] = (1 - X) * fs * Q - sig * sq * cj;
    g_chi[o] += kappa * (-B0 * Q * fs - sig * sq * ej);
  }
}

// Adds the sum of n partials (stride `stride`, k values each) to out[0..k) (k <= 3).
__global__ void k_adj_accumulate(const double* partials, int n, int stride, int k, double* out) {
  pdl_entry();
  __shared__ double scratch[3 * 32];
  double s[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    for (int j = 0; j < k; ++j) s[j] += partials[stride * i + j];
  block_reduce<3, false>(s, scratch);
  if (threadIdx.x == 0)
    for (int j = 0; j < k; ++j) out[j] += s[j];
}

}  // namespace cup
