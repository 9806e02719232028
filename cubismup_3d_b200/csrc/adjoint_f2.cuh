// Discrete adjoint of one upwind3 stage in FP32 on x-pairs of cells with
// Blackwell's packed FP32x2 arithmetic: the operator of k_adjoint_zq (SCHEME 1)
// with the structure of k_advect_zq_f2.
//
// For a stage S(f) = f + facA sum_d a_d D_d(f) + facD Lap f with the adjoint g of
// its output (see adjoint.cuh), per cell and component q:
//   out_q = g_q + facD Lap(g_q) + facA sum_d T_d(a_d g_q, |a_d| g_q)
//           + facA sum_q' g_q' D'_q(f_q')            (the adjoint of a_q, q = d)
// with, along one direction and h(o) = a(o) g(o), k(o) = |a(o)| g(o):
//   2 T = (-h-2 + 8 h-1 - 8 h+1 + h+2) + (k-2 - 4 k-1 + 6 k0 - 4 k+1 + k+2),
//   2 D'(f) = S(f) + sgn(a) Q(f),  S = f-2 - 8 f-1 + 8 f+1 - f+2,
//                                  Q = f-2 - 4 f-1 + 6 f0 - 4 f+1 + f+2,
// sgn(0) = 0 (the mean of the two one-sided slopes at the kink, as in
// up3_da). The 1/2 is folded into facA. A thread owns PPT pairs (x, x+1) of a
// TY x nx tile and marches down z: TMA ring of planes of the six fields (base
// f, adjoint input g; G = 2 halo rows), register queues of the last 5 planes
// of both, the x/y part of each plane on arrival and the z part two planes
// later; LAM: out = alpha lam + beta (...), the lam rows riding with the
// completing load. In x, the pairs at x -+ 2 come in whole and the values at
// x -+ 1 straddle two pairs, so the terms at -+1 go in as scalar FMAs.
#pragma once

#include "advect_f2.cuh"
#include "adjoint.cuh"

namespace cup {

// sgn(a) per lane: 1, -1 or 0
__device__ __forceinline__ float2 sgn2(float2 a) {
  return make_float2(a.x > 0.f ? 1.f : (a.x < 0.f ? -1.f : 0.f), a.y > 0.f ? 1.f : (a.y < 0.f ? -1.f : 0.f));
}

// 2 T along a direction whose five samples are whole pairs (y, z): the
// transport transpose from a (advecting velocity) and g at offsets -2..2.
__device__ __forceinline__ float2 tr2_pairs(float2 am2, float2 am1, float2 a0, float2 ap1, float2 ap2, float2 gm2,
                                           float2 gm1, float2 g0, float2 gp1, float2 gp2) {
  const float2 hm2 = mul2(am2, gm2), hm1 = mul2(am1, gm1), hp1 = mul2(ap1, gp1), hp2 = mul2(ap2, gp2);
  const float2 km2 = mul2(abs2(am2), gm2), km1 = mul2(abs2(am1), gm1), k0 = mul2(abs2(a0), g0);
  const float2 kp1 = mul2(abs2(ap1), gp1), kp2 = mul2(abs2(ap2), gp2);
  // (hp2 - hm2) + 8 (hm1 - hp1) + (km2 + kp2) - 4 (km1 + kp1) + 6 k0
  float2 t = add2(sub2(hp2, hm2), add2(km2, kp2));
  t = fma2(splat2(8.f), sub2(hm1, hp1), t);
  t = fma2(splat2(-4.f), add2(km1, kp1), t);
  return fma2(splat2(6.f), k0, t);
}

// S and Q of a field along a direction whose samples are whole pairs.
__device__ __forceinline__ void sq_pairs(float2 fm2, float2 fm1, float2 f0, float2 fp1, float2 fp2, float2& S,
                                         float2& Qs) {
  S = fma2(splat2(8.f), sub2(fp1, fm1), sub2(fm2, fp2));
  Qs = fma2(splat2(6.f), f0, fma2(splat2(-4.f), add2(fm1, fp1), add2(fm2, fp2)));
}

template <bool LAM, int TY, int NS, int PPT, int NXC = 0, int ZCC = 0>
constexpr size_t adjoint_f2_smem_bytes(int nx) {
  return (size_t)NS * (6 * (TY + 4) + (LAM ? 3 * TY : 0)) * nx * sizeof(float) + NS * sizeof(uint64_t);
}

// blockDim.x * PPT * 2 == TY * nx (<= 512 threads). NXC, ZCC: nx and the
// planes per work item fixed at compile time (0: read from g).
template <bool LAM, int TY, int NS, int PPT, int NXC = 0, int ZCC = 0>
__global__ void __launch_bounds__(512) k_adjoint_zq_f2(const __grid_constant__ AdjointMaps maps, const StreamGeom g,
                                                      float* __restrict__ ou, float* __restrict__ ov,
                                                      float* __restrict__ ow, float alpha, float beta, DtArg dt,
                                                      double h, double nu, double ux, double uy, double uz, int* err) {
  pdl_entry();
  constexpr int G = 2;
  constexpr int ROWS = TY + 2 * G;
  constexpr int Q = 2 * G + 1;
  constexpr int U = ZCC ? ZCC + 2 * G : 10;  // planes per unrolled chunk: a whole item, or lcm(Q, G)
  static_assert(ZCC == 0 || ZCC % 2 == 0, "items of an even plane count");
  static_assert(TY >= G, "tile height must cover the halo depth");
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  const int nx = NXC ? NXC : g.nx, ny = g.ny, nz = g.nz;
  const int zc = ZCC ? ZCC : g.zc;
  const size_t field_elems = (size_t)ROWS * nx;
  const size_t stencil_elems = 6 * field_elems;
  const size_t slot_elems = stencil_elems + (LAM ? (size_t)3 * TY * nx : 0);
  float* slots = reinterpret_cast<float*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * slot_elems * sizeof(float));
  const int tid = threadIdx.x;
  const int PL = zc + 2 * G;
  const int my_items = blockIdx.x < g.n_items ? (g.n_items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int L = my_items * PL;
  const uint32_t stencil_bytes = (uint32_t)(stencil_elems * sizeof(float));
  const uint32_t lam_bytes = (uint32_t)(3 * TY * nx * sizeof(float));

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto issue = [&](int q) {
    const int it = q / PL, j = q - it * PL;
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY, z0 = zi * zc;
    int z = z0 - G + j;
    z = z < 0 ? z + nz : (z >= nz ? z - nz : z);
    const int s = q % NS;
    float* dst = slots + s * slot_elems;
    int ylo = y0 - G;
    if (ylo < 0) ylo += ny;
    int yhi = y0 + TY;
    if (yhi >= ny) yhi -= ny;
    const bool with_lam = LAM && j >= 2 * G;
    mbar_arrive_expect_tx(&full[s], stencil_bytes + (with_lam ? lam_bytes : 0u));
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      float* fd = dst + f * field_elems;
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
  const int half = nx >> 1;
  int px[PPT], cy[PPT];
  int ctr[PPT], xl[PPT], xr[PPT];  // slot offsets: the pair, the pairs at x -+ 2
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int pi = tid + i * blockDim.x;
    px[i] = (pi % half) * 2;
    cy[i] = pi / half;
    ctr[i] = (G + cy[i]) * nx + px[i];
    xl[i] = (G + cy[i]) * nx + ((px[i] - 2) & mask);
    xr[i] = (G + cy[i]) * nx + ((px[i] + 2) & mask);
  }
  const size_t plane = (size_t)nx * ny;
  const double dtv = dt.get();
  const float2 facA = splat2((float)(-dtv / (12 * h)));  // facA of the stage with the 1/2 of T and D' folded in
  const float2 facD = splat2((float)((nu / h) * (dtv / h)));
  const float2 uinf[3] = {splat2((float)ux), splat2((float)uy), splat2((float)uz)};
  const float2 alpha2 = splat2(alpha), beta2 = splat2(beta);

  float2 qf[3][Q][PPT];  // base field pairs, plane j in slot j % Q
  float2 qg[3][Q][PPT];  // adjoint input pairs
  float2 part[3][G][PPT];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int d = 0; d < Q; ++d)
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
        qf[f][d][i] = splat2(0.f);
        qg[f][d][i] = splat2(0.f);
      }
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int d = 0; d < G; ++d)
#pragma unroll
      for (int i = 0; i < PPT; ++i) part[f][d][i] = splat2(0.f);

  bool ok = true;
  int q = 0;
  for (int it = 0; it < my_items; ++it) {
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY, z0 = zi * zc;
    size_t obase[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) obase[i] = gidx(px[i], y0 + cy[i], z0, nx, ny);
    for (int j0 = 0; j0 < PL; j0 += U) {
#pragma unroll
      for (int jj = 0; jj < U; ++jj) {
        const int j = j0 + jj;
        if (j >= PL) break;
        const int s = q % NS;
        if (ok) ok = mbar_wait(&full[s], (q / NS) & 1, err);
        if (ok) {
          const float* sl = slots + s * slot_elems;
          const int QN = jj % Q;
#pragma unroll
          for (int f = 0; f < 3; ++f)
#pragma unroll
            for (int i = 0; i < PPT; ++i) {
              qf[f][QN][i] = *reinterpret_cast<const float2*>(sl + f * field_elems + ctr[i]);
              qg[f][QN][i] = *reinterpret_cast<const float2*>(sl + (3 + f) * field_elems + ctr[i]);
            }
          // z terms and output of plane k = j - 2G
          if (j >= 2 * G) {
            const int k = j - 2 * G;
            const int QC = (jj + 3 * Q - G) % Q;
            const int QM1 = (jj + 3 * Q - G - 1) % Q, QP1 = (jj + 3 * Q - G + 1) % Q;
            const int QM2 = (jj + 3 * Q - G - 2) % Q, QP2 = (jj + 3 * Q - G + 2) % Q;
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const size_t o = obase[i] + (size_t)k * plane;
              const float2 am2 = add2(qf[2][QM2][i], uinf[2]), am1 = add2(qf[2][QM1][i], uinf[2]);
              const float2 a0 = add2(qf[2][QC][i], uinf[2]);
              const float2 ap1 = add2(qf[2][QP1][i], uinf[2]), ap2 = add2(qf[2][QP2][i], uinf[2]);
              // adjoint of a_z at the cell: sum_q' g_q' D'_z(f_q')
              float2 sS = splat2(0.f), sQ = splat2(0.f);
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                float2 S, Qs;
                sq_pairs(qf[f][QM2][i], qf[f][QM1][i], qf[f][QC][i], qf[f][QP1][i], qf[f][QP2][i], S, Qs);
                sS = fma2(qg[f][QC][i], S, sS);
                sQ = fma2(qg[f][QC][i], Qs, sQ);
              }
              const float2 advz = fma2(sgn2(a0), sQ, sS);
              float2 outv[3];
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const float2 g0 = qg[f][QC][i];
                const float2 tz = tr2_pairs(am2, am1, a0, ap1, ap2, qg[f][QM2][i], qg[f][QM1][i], g0,
                                            qg[f][QP1][i], qg[f][QP2][i]);
                // Lap_z with the centre's -6 g0
                const float2 lz = fma2(splat2(-6.f), g0, add2(qg[f][QM1][i], qg[f][QP1][i]));
                float2 v = fma2(facD, lz, fma2(facA, tz, part[f][PS][i]));
                if (f == 2) v = fma2(facA, advz, v);
                outv[f] = v;
              }
              if constexpr (LAM) {
                const float* ls = sl + stencil_elems + cy[i] * nx + px[i];
#pragma unroll
                for (int f = 0; f < 3; ++f)
                  outv[f] = fma2(alpha2, *reinterpret_cast<const float2*>(ls + f * TY * nx), mul2(beta2, outv[f]));
              } else {
#pragma unroll
                for (int f = 0; f < 3; ++f) outv[f] = mul2(beta2, outv[f]);
              }
              *reinterpret_cast<float2*>(ou + o) = outv[0];
              *reinterpret_cast<float2*>(ov + o) = outv[1];
              *reinterpret_cast<float2*>(ow + o) = outv[2];
            }
          }
          // x/y part of plane j
          if (j >= G && j < G + zc) {
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const float* Fx = sl;                // base u (advects in x)
              const float* Fy = sl + field_elems;  // base v (advects in y)
              const int c = ctr[i];
              // advecting velocities: x at x-2..x+3 (pairs A, C, B), y at rows -2..2
              const float2 axA = add2(*reinterpret_cast<const float2*>(Fx + xl[i]), uinf[0]);
              const float2 axC = add2(qf[0][QN][i], uinf[0]);
              const float2 axB = add2(*reinterpret_cast<const float2*>(Fx + xr[i]), uinf[0]);
              const float2 aym2 = add2(*reinterpret_cast<const float2*>(Fy + c - 2 * nx), uinf[1]);
              const float2 aym1 = add2(*reinterpret_cast<const float2*>(Fy + c - nx), uinf[1]);
              const float2 ay0 = add2(qf[1][QN][i], uinf[1]);
              const float2 ayp1 = add2(*reinterpret_cast<const float2*>(Fy + c + nx), uinf[1]);
              const float2 ayp2 = add2(*reinterpret_cast<const float2*>(Fy + c + 2 * nx), uinf[1]);
              const float2 kxA = abs2(axA), kxC = abs2(axC), kxB = abs2(axB);
              // adjoints of a_x, a_y at the cell: sum_q' g_q' D'(f_q'), as S and Q sums
              float2 sSx = splat2(0.f), sQx = splat2(0.f), sSy = splat2(0.f), sQy = splat2(0.f);
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const float* F = sl + f * field_elems;
                const float2 fA = *reinterpret_cast<const float2*>(F + xl[i]);
                const float2 fC = qf[f][QN][i];
                const float2 fB = *reinterpret_cast<const float2*>(F + xr[i]);
                const float2 gq = qg[f][QN][i];
                // x: S = f-2 - 8 f-1 + 8 f+1 - f+2, Q = f-2 - 4 f-1 + 6 f0 - 4 f+1 + f+2
                float2 Sx = sub2(fA, fB);  // the -+2 terms of each lane
                Sx.x = fmaf(8.f, fC.y - fA.y, Sx.x);
                Sx.y = fmaf(8.f, fB.x - fC.x, Sx.y);
                float2 Qx = fma2(splat2(6.f), fC, add2(fA, fB));
                Qx.x = fmaf(-4.f, fA.y + fC.y, Qx.x);
                Qx.y = fmaf(-4.f, fC.x + fB.x, Qx.y);
                float2 Sy, Qy;
                sq_pairs(*reinterpret_cast<const float2*>(F + c - 2 * nx), *reinterpret_cast<const float2*>(F + c - nx),
                         fC, *reinterpret_cast<const float2*>(F + c + nx),
                         *reinterpret_cast<const float2*>(F + c + 2 * nx), Sy, Qy);
                sSx = fma2(gq, Sx, sSx);
                sQx = fma2(gq, Qx, sQx);
                sSy = fma2(gq, Sy, sSy);
                sQy = fma2(gq, Qy, sQy);
              }
              const float2 advx = fma2(sgn2(axC), sQx, sSx);
              const float2 advy = fma2(sgn2(ay0), sQy, sSy);
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const float* Gf = sl + (3 + f) * field_elems;
                const float2 gA = *reinterpret_cast<const float2*>(Gf + xl[i]);
                const float2 g0 = qg[f][QN][i];
                const float2 gB = *reinterpret_cast<const float2*>(Gf + xr[i]);
                const float2 gym2 = *reinterpret_cast<const float2*>(Gf + c - 2 * nx);
                const float2 gym1 = *reinterpret_cast<const float2*>(Gf + c - nx);
                const float2 gyp1 = *reinterpret_cast<const float2*>(Gf + c + nx);
                const float2 gyp2 = *reinterpret_cast<const float2*>(Gf + c + 2 * nx);
                // x transport: products of the pairs, then the -+2 terms as pairs and the -+1 terms per lane
                const float2 hA = mul2(axA, gA), hC = mul2(axC, g0), hB = mul2(axB, gB);
                const float2 kA = mul2(kxA, gA), kC = mul2(kxC, g0), kB = mul2(kxB, gB);
                // lane x: -hA.x + 8 hA.y - 8 hC.y + hB.x + kA.x - 4 kA.y + 6 kC.x - 4 kC.y + kB.x
                // lane x+1: -hA.y + 8 hC.x - 8 hB.x + hB.y + kA.y - 4 kC.x + 6 kC.y - 4 kB.x + kB.y
                float2 tx = fma2(splat2(6.f), kC, add2(sub2(hB, hA), add2(kA, kB)));
                tx.x = fmaf(8.f, hA.y - hC.y, fmaf(-4.f, kA.y + kC.y, tx.x));
                tx.y = fmaf(8.f, hC.x - hB.x, fmaf(-4.f, kC.x + kB.x, tx.y));
                const float2 ty = tr2_pairs(aym2, aym1, ay0, ayp1, ayp2, gym2, gym1, g0, gyp1, gyp2);
                // Lap in x and y without the centre (the z part adds -6 g0)
                float2 lxy = add2(add2(gym1, gyp1), make_float2(gA.y + g0.y, g0.x + gB.x));
                float2 v = fma2(facD, lxy, fma2(facA, add2(tx, ty), g0));
                if (f == 0) v = fma2(facA, advx, v);
                if (f == 1) v = fma2(facA, advy, v);
                part[f][PS][i] = v;
              }
            }
          }
        }
        __syncthreads();  // slot s fully consumed
        if (tid == 0 && ok && q_issued < L && q_issued == q + NS) issue(q_issued++);
        ++q;
      }
    }
  }
  // after a timed-out wait: bounded drain of the loads that may be in flight
  if (!ok && tid == 0) {
    for (int r = q_issued - NS < 0 ? 0 : q_issued - NS; r < q_issued; ++r)
      mbar_wait(&full[r % NS], (r / NS) & 1, nullptr);
  }
}

}  // namespace cup
