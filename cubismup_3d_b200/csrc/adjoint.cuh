// Discrete adjoint of one explicit advection-diffusion stage
// S(f) = f + facA sum_d a_d D_d(f) + facD Lap(f), a_d = f_d + uinf_d, the stage
// of KernelAdvectDiffuse (source/operators/AdvectionDiffusion.cpp:111-144) or
// of the upwind3 + RK2 scheme. The reference has no adjoint; this is new.
//
// For upwind3, a D(f) with the sign-selected stencil equals
// 1/2 (a S(f) + |a| Q(f)), S(f) = f-2 - 8f-1 + 8f+1 - f+2 (antisymmetric) and
// Q(f) = f-2 - 4f-1 + 6f0 - 4f+1 + f+2 (symmetric), so with the signs frozen at
// the base state the transpose of the transport part is
// 1/2 (-S(a g) + Q(|a| g)): a stencil of point-wise products, no scatter.
// For the central scheme a D(f) = a (f+1 - f-1) and its transpose is
// (a g)-1 - (a g)+1. With g the adjoint of the stage output:
//   S'(f)^T g = g + facD Lap(g) + facA sum_d T_d^T(a_d g)
//               + facA e_q sum_q' g_q' D_q(f_q')        (a_q's own adjoint)
// and the kernel writes out = alpha lam + beta S'(f)^T g (lam point-wise).
//
// Structure as k_advect_zq: TMA ring of planes (base f and g with G halo
// rows, lam's output rows riding with the completing load), register queues
// of the last 2G+1 planes of f and g, x/y partials on arrival, z terms at
// output, one block barrier per plane.
#pragma once

#include "advect.cuh"

namespace cup {

struct AdjointMaps {
  CUtensorMap main[6];  // f (3) then g (3), box {nx, TY, 1}
  CUtensorMap halo[6];  // box {nx, G, 1}
  CUtensorMap lam[3];   // point-wise lam, box {nx, TY, 1}
};

template <typename T, int SCHEME, bool LAM, int TY, int NS, int CPT>
constexpr size_t adjoint_smem_bytes(int nx) {
  constexpr int G = SCHEME == 0 ? 1 : 2;
  return (size_t)NS * (6 * (TY + 2 * G) + (LAM ? 3 * TY : 0)) * nx * sizeof(T) + NS * sizeof(uint64_t);
}

// transpose of the transport stencil at one point from the 5 products
// h(o) = a(o) g(o) and k(o) = |a(o)| g(o), o = -2..2 (upwind3) or the 2 products
// h(-1), h(+1) (central).
template <typename T>
__device__ __forceinline__ T tabs(T x) {
  return x < (T)0 ? -x : x;
}

// Derivative of a up3(a; f) with respect to a (the adjoint of the advecting
// velocity): up3(a; f) off a = 0; at a = 0, where the one-sided derivatives
// are the two upwind stencils, their mean (f-2 - 8 f-1 + 8 f+1 - f+2) / 2, the
// value central differences see (a flow started from rest has a_y = a_z = 0
// in every cell of its first step).
template <typename T>
__device__ __forceinline__ T up3_da(T a, T fm2, T fm1, T f0, T fp1, T fp2) {
  if (a == (T)0) return (T)0.5 * (fm2 - (T)8 * fm1 + (T)8 * fp1 - fp2);
  return up3(a, fm2, fm1, f0, fp1, fp2);
}

template <typename T>
__device__ __forceinline__ T tr_up3(T hm2, T hm1, T hp1, T hp2, T km2, T km1, T k0, T kp1, T kp2) {
  return (T)0.5 * ((-hm2 + (T)8 * hm1 - (T)8 * hp1 + hp2) + (km2 - (T)4 * km1 + (T)6 * k0 - (T)4 * kp1 + kp2));
}

template <typename T, int SCHEME, bool LAM, int TY, int NS, int CPT>
__global__ void __launch_bounds__(512) k_adjoint_zq(const __grid_constant__ AdjointMaps maps, const StreamGeom g,
                                                   T* __restrict__ ou, T* __restrict__ ov, T* __restrict__ ow,
                                                   T alpha, T beta, DtArg dt, double h, double nu, double ux,
                                                   double uy, double uz, int* err) {
  pdl_entry();
  constexpr int G = SCHEME == 0 ? 1 : 2;
  constexpr int ROWS = TY + 2 * G;
  constexpr int Q = 2 * G + 1;
  constexpr int U = (G == 1) ? 3 : 10;
  // a G-row halo box starting at y0 - G (wrapped) stays inside [0, ny) only if y0 is a multiple of TY >= G
  static_assert(TY >= G, "tile height must cover the halo depth");
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t field_elems = (size_t)ROWS * nx;
  const size_t stencil_elems = 6 * field_elems;
  const size_t slot_elems = stencil_elems + (LAM ? (size_t)3 * TY * nx : 0);
  T* slots = reinterpret_cast<T*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * slot_elems * sizeof(T));
  const int tid = threadIdx.x;
  const int PL = g.zc + 2 * G;
  const int my_items = blockIdx.x < g.n_items ? (g.n_items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int L = my_items * PL;
  const uint32_t stencil_bytes = (uint32_t)(stencil_elems * sizeof(T));
  const uint32_t lam_bytes = (uint32_t)(3 * TY * nx * sizeof(T));

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto issue = [&](int q) {
    const int it = q / PL, j = q - it * PL;
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY, z0 = zi * g.zc;
    int z = z0 - G + j;
    z = z < 0 ? z + nz : (z >= nz ? z - nz : z);
    const int s = q % NS;
    T* dst = slots + s * slot_elems;
    int ylo = y0 - G;
    if (ylo < 0) ylo += ny;
    int yhi = y0 + TY;
    if (yhi >= ny) yhi -= ny;
    const bool with_lam = LAM && j >= 2 * G;
    mbar_arrive_expect_tx(&full[s], stencil_bytes + (with_lam ? lam_bytes : 0u));
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      T* fd = dst + f * field_elems;
      tma_load_3d(fd, &maps.halo[f], 0, ylo, z, &full[s]);
      tma_load_3d(fd + G * nx, &maps.main[f], 0, y0, z, &full[s]);
      tma_load_3d(fd + (G + TY) * nx, &maps.halo[f], 0, yhi, z, &full[s]);
    }
    if (with_lam) {
      const int zk = z0 + (j - 2 * G);
#pragma unroll
      for (int f = 0; f < 3; ++f) tma_load_3d(dst + stencil_elems + f * TY * nx, &maps.lam[f], 0, y0, zk, &full[s]);
    }
  };

  int q_issued = 0;
  if (tid == 0)
    for (; q_issued < min(L, NS); ++q_issued) issue(q_issued);

  const int mask = nx - 1;
  int cx[CPT], cy[CPT];
#pragma unroll
  for (int i = 0; i < CPT; ++i) {
    const int c = tid + i * blockDim.x;
    cx[i] = c & mask;
    cy[i] = c >> g.log2nx;
  }
  const double dtv = dt.get();
  const T facA = (T)(SCHEME == 0 ? -dtv / (2 * h) : -dtv / (6 * h));
  const T facD = (T)((nu / h) * (dtv / h));
  const T uinf[3] = {(T)ux, (T)uy, (T)uz};

  T qf[3][Q][CPT];  // base field centre values, plane j in slot j % Q
  T qg[3][Q][CPT];  // adjoint input centre values
  T part[3][G][CPT];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int d = 0; d < Q; ++d)
#pragma unroll
      for (int i = 0; i < CPT; ++i) {
        qf[f][d][i] = (T)0;
        qg[f][d][i] = (T)0;
      }
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int d = 0; d < G; ++d)
#pragma unroll
      for (int i = 0; i < CPT; ++i) part[f][d][i] = (T)0;

  bool ok = true;
  int q = 0;
  for (int it = 0; it < my_items; ++it) {
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY, z0 = zi * g.zc;
    for (int j0 = 0; j0 < PL; j0 += U) {
#pragma unroll
      for (int jj = 0; jj < U; ++jj) {
        const int j = j0 + jj;
        const int s = q % NS;
        if (ok) ok = mbar_wait(&full[s], (q / NS) & 1, err);
        if (ok) {
          const T* sl = slots + s * slot_elems;
          const int QN = jj % Q;
#pragma unroll
          for (int f = 0; f < 3; ++f)
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
              const int off = (G + cy[i]) * nx + cx[i];
              qf[f][QN][i] = sl[f * field_elems + off];
              qg[f][QN][i] = sl[(3 + f) * field_elems + off];
            }
          // z terms and output of plane k = j - 2G
          if (j >= 2 * G) {
            const int k = j - 2 * G;
            const int QC = (jj + 3 * Q - G) % Q;
            const int QM1 = (jj + 3 * Q - G - 1) % Q, QP1 = (jj + 3 * Q - G + 1) % Q;
            const int QM2 = (jj + 3 * Q - G - 2) % Q, QP2 = (jj + 3 * Q - G + 2) % Q;
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
              const size_t o = gidx(cx[i], y0 + cy[i], z0 + k, nx, ny);
              const T azc = qf[2][QC][i] + uinf[2];
              // adjoint of a_z at the cell: sum_q' g_q' D_z(f_q')
              T advz = (T)0;
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                T dz;
                if constexpr (SCHEME == 0) dz = qf[f][QP1][i] - qf[f][QM1][i];
                else dz = up3_da(azc, qf[f][QM2][i], qf[f][QM1][i], qf[f][QC][i], qf[f][QP1][i], qf[f][QP2][i]);
                advz += qg[f][QC][i] * dz;
              }
              T outv[3];
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const T g0 = qg[f][QC][i];
                T tz;
                if constexpr (SCHEME == 0) {
                  tz = (qf[2][QM1][i] + uinf[2]) * qg[f][QM1][i] - (qf[2][QP1][i] + uinf[2]) * qg[f][QP1][i];
                } else {
                  const T am2 = qf[2][QM2][i] + uinf[2], am1 = qf[2][QM1][i] + uinf[2];
                  const T ap1 = qf[2][QP1][i] + uinf[2], ap2 = qf[2][QP2][i] + uinf[2];
                  tz = tr_up3(am2 * qg[f][QM2][i], am1 * qg[f][QM1][i], ap1 * qg[f][QP1][i], ap2 * qg[f][QP2][i],
                              tabs(am2) * qg[f][QM2][i], tabs(am1) * qg[f][QM1][i], tabs(azc) * g0,
                              tabs(ap1) * qg[f][QP1][i], tabs(ap2) * qg[f][QP2][i]);
                }
                T v = part[f][PS][i] + facD * (qg[f][QM1][i] + qg[f][QP1][i] - g0 * 6) + facA * tz;
                if (f == 2) v += facA * advz;
                outv[f] = v;
              }
              if constexpr (LAM) {
                const T* ls = sl + stencil_elems + cy[i] * nx + cx[i];
                ou[o] = alpha * ls[0] + beta * outv[0];
                ov[o] = alpha * ls[TY * nx] + beta * outv[1];
                ow[o] = alpha * ls[2 * TY * nx] + beta * outv[2];
              } else {
                ou[o] = beta * outv[0];
                ov[o] = beta * outv[1];
                ow[o] = beta * outv[2];
              }
            }
          }
          // x/y partial of plane j
          if (j >= G && j < G + g.zc) {
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
              const int x = cx[i], r = G + cy[i];
              const int xm1 = (x - 1) & mask, xp1 = (x + 1) & mask, xm2 = (x - 2) & mask, xp2 = (x + 2) & mask;
              const T* Fx = sl;                    // base u (advects in x)
              const T* Fy = sl + field_elems;      // base v (advects in y)
              const T ax0 = qf[0][QN][i] + uinf[0], ay0 = qf[1][QN][i] + uinf[1];
              // adjoints of a_x, a_y at the cell: sum_q' g_q' D(f_q')
              T advx = (T)0, advy = (T)0;
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const T* F = sl + f * field_elems;
                const T f0 = qf[f][QN][i], gq = qg[f][QN][i];
                T dx, dy;
                if constexpr (SCHEME == 0) {
                  dx = F[r * nx + xp1] - F[r * nx + xm1];
                  dy = F[(r + 1) * nx + x] - F[(r - 1) * nx + x];
                } else {
                  dx = up3_da(ax0, F[r * nx + xm2], F[r * nx + xm1], f0, F[r * nx + xp1], F[r * nx + xp2]);
                  dy = up3_da(ay0, F[(r - 2) * nx + x], F[(r - 1) * nx + x], f0, F[(r + 1) * nx + x], F[(r + 2) * nx + x]);
                }
                advx += gq * dx;
                advy += gq * dy;
              }
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const T* Gf = sl + (3 + f) * field_elems;
                const T g0 = qg[f][QN][i];
                const T gxm1 = Gf[r * nx + xm1], gxp1 = Gf[r * nx + xp1];
                const T gym1 = Gf[(r - 1) * nx + x], gyp1 = Gf[(r + 1) * nx + x];
                T tx, ty;
                if constexpr (SCHEME == 0) {
                  tx = (Fx[r * nx + xm1] + uinf[0]) * gxm1 - (Fx[r * nx + xp1] + uinf[0]) * gxp1;
                  ty = (Fy[(r - 1) * nx + x] + uinf[1]) * gym1 - (Fy[(r + 1) * nx + x] + uinf[1]) * gyp1;
                } else {
                  const T gxm2 = Gf[r * nx + xm2], gxp2 = Gf[r * nx + xp2];
                  const T gym2 = Gf[(r - 2) * nx + x], gyp2 = Gf[(r + 2) * nx + x];
                  const T axm2 = Fx[r * nx + xm2] + uinf[0], axm1 = Fx[r * nx + xm1] + uinf[0];
                  const T axp1 = Fx[r * nx + xp1] + uinf[0], axp2 = Fx[r * nx + xp2] + uinf[0];
                  const T aym2 = Fy[(r - 2) * nx + x] + uinf[1], aym1 = Fy[(r - 1) * nx + x] + uinf[1];
                  const T ayp1 = Fy[(r + 1) * nx + x] + uinf[1], ayp2 = Fy[(r + 2) * nx + x] + uinf[1];
                  tx = tr_up3(axm2 * gxm2, axm1 * gxm1, axp1 * gxp1, axp2 * gxp2, tabs(axm2) * gxm2,
                              tabs(axm1) * gxm1, tabs(ax0) * g0, tabs(axp1) * gxp1, tabs(axp2) * gxp2);
                  ty = tr_up3(aym2 * gym2, aym1 * gym1, ayp1 * gyp1, ayp2 * gyp2, tabs(aym2) * gym2,
                              tabs(aym1) * gym1, tabs(ay0) * g0, tabs(ayp1) * gyp1, tabs(ayp2) * gyp2);
                }
                T v = g0 + facD * (gyp1 + gym1 + gxp1 + gxm1) + facA * (tx + ty);
                if (f == 0) v += facA * advx;
                if (f == 1) v += facA * advy;
                part[f][PS][i] = v;
              }
            }
          }
        }
        __syncthreads();
        if (tid == 0 && ok && q_issued < L && q_issued == q + NS) issue(q_issued++);
        ++q;
      }
    }
  }
  if (!ok && tid == 0) {
    for (int r = q - NS < 0 ? 0 : q - NS; r < q_issued; ++r) mbar_wait(&full[r % NS], (r / NS) & 1, nullptr);
  }
}

}  // namespace cup
