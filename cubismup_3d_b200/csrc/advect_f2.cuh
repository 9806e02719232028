// FP32 upwind3 + RK2 stages with Blackwell's packed FP32x2 arithmetic.
//
// Same streaming structure as k_advect_zq (TMA ring of planes, register
// z-queues, x/y part on arrival, one block barrier per plane), but each
// thread owns PPT pairs of x-adjacent cells and every arithmetic instruction
// works on a pair (fma/add/mul .f32x2). The upwind term uses the branch-free
// identity
//   a up3(a; f) = 1/2 (a S(f) + |a| Q(f)),
//   S = f-2 - 8 f-1 + 8 f+1 - f+2,  Q = f-2 - 4 f-1 + 6 f0 - 4 f+1 + f+2,
// which is the same operator as the sign-selected stencil (at a = 0 both
// give 0), so both cells of a pair follow one instruction stream.
#pragma once

#include "advect.cuh"

namespace cup {

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 abs2(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }

// The five weights of one direction of the update, for a pair: with
// facA = -dt / (12 h) and facD = nu dt / h^2,
//   facA (a S(f) + |a| Q(f)) + facD (f-1 + f+1 - 2 f0) = m2 f-2 + m1 f-1 + c0 f0 + p1 f+1 + p2 f+2,
//   m2 = A1 + A2, p2 = A2 - A1, m1 = -8 A1 - 4 A2 + facD, p1 = 8 A1 - 4 A2 + facD,
//   c0 = 6 A2 - 2 facD,  A1 = facA a, A2 = facA |a|.
// They depend on the advecting velocity only, so the three components of a
// cell share them (five FMAs per component and direction).
struct Weights5 {
  float2 m2, m1, c0, p1, p2;
};
__device__ __forceinline__ Weights5 weights5(float2 a, float2 facA, float2 facD, float2 m2FacD) {
  const float2 A1 = mul2(facA, a), A2 = mul2(facA, abs2(a));
  const float2 t = fma2(splat2(-4.f), A2, facD);
  Weights5 k;
  k.m2 = add2(A1, A2);
  k.p2 = sub2(A2, A1);
  k.m1 = fma2(splat2(-8.f), A1, t);
  k.p1 = fma2(splat2(8.f), A1, t);
  k.c0 = fma2(splat2(6.f), A2, m2FacD);
  return k;
}
__device__ __forceinline__ float2 apply5(const Weights5& k, float2 fm2, float2 fm1, float2 f0, float2 fp1, float2 fp2,
                                         float2 acc) {
  return fma2(k.m2, fm2, fma2(k.m1, fm1, fma2(k.c0, f0, fma2(k.p1, fp1, fma2(k.p2, fp2, acc)))));
}
__device__ __forceinline__ float2 apply5(const Weights5& k, float2 fm2, float2 fm1, float2 f0, float2 fp1, float2 fp2) {
  return fma2(k.m2, fm2, fma2(k.m1, fm1, fma2(k.c0, f0, fma2(k.p1, fp1, mul2(k.p2, fp2)))));
}

// STAGE2 false: out = f + dt A(f); true: out = 1/2 (f^n + f1 + dt A(f1)).
// blockDim.x * PPT * 2 == TY * nx (<= 512 threads).
// NXC, ZCC: nx and the planes per work item fixed at compile time (0: read
// from g). Fixed, every shared-memory offset of the stencil is an immediate
// on a per-thread base register and each item's planes unroll completely
// (ring slot and z-queue position known per plane).
template <bool STAGE2, int TY, int NS, int PPT, int NXC = 0, int ZCC = 0>
__global__ void __launch_bounds__(512) k_advect_zq_f2(const __grid_constant__ AdvectMaps maps, const StreamGeom g,
                                                     float* __restrict__ ou, float* __restrict__ ov,
                                                     float* __restrict__ ow, DtArg dt, double h, double nu, double ux,
                                                     double uy, double uz, int* err) {
  pdl_entry();
  constexpr int G = 2;
  constexpr int ROWS = TY + 2 * G;
  constexpr int Q = 2 * G + 1;
  constexpr int U = ZCC ? ZCC + 2 * G : 10;  // planes per unrolled chunk: a whole item, or lcm(Q, G)
  constexpr bool SLOT_CT = ZCC != 0 && (ZCC + 2 * G) % NS == 0;  // ring slot of plane j is j % NS
  static_assert(ZCC == 0 || ZCC % 2 == 0, "paired barriers need an even plane count");
  static_assert(TY >= G, "tile height must cover the halo depth");
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  const int nx = NXC ? NXC : g.nx, ny = g.ny, nz = g.nz;
  const int zc = ZCC ? ZCC : g.zc;
  const size_t field_elems = (size_t)ROWS * nx;
  const size_t stencil_elems = 3 * field_elems;
  const size_t slot_elems = stencil_elems + (STAGE2 ? (size_t)3 * TY * nx : 0);
  float* slots = reinterpret_cast<float*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * slot_elems * sizeof(float));
  const int tid = threadIdx.x;
  const int PL = zc + 2 * G;
  const int my_items = blockIdx.x < g.n_items ? (g.n_items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int L = my_items * PL;
  const uint32_t stencil_bytes = (uint32_t)(stencil_elems * sizeof(float));
  const uint32_t base_bytes = (uint32_t)(3 * TY * nx * sizeof(float));

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
    const bool with_base = STAGE2 && j >= 2 * G;
    mbar_arrive_expect_tx(&full[s], stencil_bytes + (with_base ? base_bytes : 0u));
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      float* fd = dst + f * field_elems;
      tma_load_3d(fd, &maps.halo[f], 0, ylo, z, &full[s]);
      tma_load_3d(fd + G * nx, &maps.main[f], 0, y0, z, &full[s]);
      tma_load_3d(fd + (G + TY) * nx, &maps.halo[f], 0, yhi, z, &full[s]);
    }
    if (with_base) {
      const int zk = z0 + (j - 2 * G);
#pragma unroll
      for (int f = 0; f < 3; ++f) tma_load_3d(dst + stencil_elems + f * TY * nx, &maps.base[f], 0, y0, zk, &full[s]);
    }
  };

  int q_issued = 0;
  if (tid == 0)
    for (; q_issued < min(L, NS); ++q_issued) issue(q_issued);

  const int mask = nx - 1;
  const int half = nx >> 1;
  int px[PPT], cy[PPT];  // even x of the pair, tile row
  int ctr[PPT], xl[PPT], xr[PPT];  // slot offsets: centre row, pairs at x -+ 2 in that row
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
  const float2 facA = splat2((float)(-dtv / (12 * h)));  // the 1/2 of the symmetric form folded in
  const float2 facD = splat2((float)((nu / h) * (dtv / h)));
  const float2 m2facD = splat2(-2.f * (float)((nu / h) * (dtv / h)));
  const float2 uinf[3] = {splat2((float)ux), splat2((float)uy), splat2((float)uz)};

  float2 qv[3][Q][PPT];
  float2 part[3][G][PPT];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int d = 0; d < Q; ++d)
#pragma unroll
      for (int i = 0; i < PPT; ++i) qv[f][d][i] = splat2(0.f);
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
    size_t obase[PPT];  // output index of the pair in plane z0
#pragma unroll
    for (int i = 0; i < PPT; ++i) obase[i] = gidx(px[i], y0 + cy[i], z0, nx, ny);
    const int q0 = q;  // first load of the item (a multiple of NS when SLOT_CT)
    for (int j0 = 0; j0 < PL; j0 += U) {
#pragma unroll
      for (int jj = 0; jj < U; ++jj) {
        const int j = j0 + jj;
        if (j >= PL) break;  // items of PL planes, PL not a multiple of U (zc = 8)
        const int s = SLOT_CT ? jj % NS : q % NS;
        const uint32_t phase = SLOT_CT ? ((q0 / NS + jj / NS) & 1) : ((q / NS) & 1);
        if (ok) ok = mbar_wait(&full[s], phase, err);
        if (ok) {
          const float* sl = slots + s * slot_elems;
          const int QN = jj % Q;
#pragma unroll
          for (int f = 0; f < 3; ++f)
#pragma unroll
            for (int i = 0; i < PPT; ++i)
              qv[f][QN][i] = *reinterpret_cast<const float2*>(sl + f * field_elems + ctr[i]);
          if (j >= 2 * G) {
            const int k = j - 2 * G;
            const int QC = (jj + 3 * Q - G) % Q;
            const int QM1 = (jj + 3 * Q - G - 1) % Q, QP1 = (jj + 3 * Q - G + 1) % Q;
            const int QM2 = (jj + 3 * Q - G - 2) % Q, QP2 = (jj + 3 * Q - G + 2) % Q;
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const size_t o = obase[i] + (size_t)k * plane;
              const Weights5 kz = weights5(add2(qv[2][QC][i], uinf[2]), facA, facD, m2facD);
              float2 outv[3];
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const float2 f0 = qv[f][QC][i];
                outv[f] = apply5(kz, qv[f][QM2][i], qv[f][QM1][i], f0, qv[f][QP1][i], qv[f][QP2][i],
                                 add2(f0, part[f][PS][i]));
              }
              if constexpr (STAGE2) {
                const float* bs = sl + stencil_elems + cy[i] * nx + px[i];
#pragma unroll
                for (int f = 0; f < 3; ++f)
                  outv[f] = mul2(splat2(0.5f), add2(*reinterpret_cast<const float2*>(bs + f * TY * nx), outv[f]));
              }
              *reinterpret_cast<float2*>(ou + o) = outv[0];
              *reinterpret_cast<float2*>(ov + o) = outv[1];
              *reinterpret_cast<float2*>(ow + o) = outv[2];
            }
          }
          if (j >= G && j < G + zc) {
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const Weights5 kx = weights5(add2(qv[0][QN][i], uinf[0]), facA, facD, m2facD);
              const Weights5 ky = weights5(add2(qv[1][QN][i], uinf[1]), facA, facD, m2facD);
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const float* F = sl + f * field_elems;
                const float* Fc = F + ctr[i];
                const float2 c0 = qv[f][QN][i];
                const float2 A = *reinterpret_cast<const float2*>(F + xl[i]);
                const float2 B = *reinterpret_cast<const float2*>(F + xr[i]);
                const float2 ym2 = *reinterpret_cast<const float2*>(Fc - 2 * nx);
                const float2 ym1 = *reinterpret_cast<const float2*>(Fc - nx);
                const float2 yp1 = *reinterpret_cast<const float2*>(Fc + nx);
                const float2 yp2 = *reinterpret_cast<const float2*>(Fc + 2 * nx);
                // x: the pairs at x -+ 1 straddle A|c0 and c0|B, so their two
                // weights go in as scalar FMAs (no register shuffle)
                float2 acc = fma2(kx.m2, A, fma2(kx.c0, c0, fma2(kx.p2, B, apply5(ky, ym2, ym1, c0, yp1, yp2))));
                acc.x = fmaf(kx.m1.x, A.y, fmaf(kx.p1.x, c0.y, acc.x));
                acc.y = fmaf(kx.m1.y, c0.x, fmaf(kx.p1.y, B.x, acc.y));
                part[f][PS][i] = acc;
              }
            }
          }
        }
        // rings of 4+ slots: one block barrier per two planes (slots of loads
        // q-1 and q fully consumed, refill both; q is odd here: PL and U are
        // even); shallower rings keep one barrier per plane for lookahead
        if constexpr (NS >= 4) {
          if (jj & 1) {
            __syncthreads();
            if (tid == 0 && ok)
              for (int r = q - 1 + NS; r <= q + NS && r < L; ++r)
                if (r == q_issued) issue(q_issued++);
          }
        } else {
          __syncthreads();  // slot s fully consumed
          if (tid == 0 && ok && q_issued < L && q_issued == q + NS) issue(q_issued++);
        }
        ++q;
      }
    }
  }
  // after a timed-out wait: bounded drain of the loads that may be in flight
  // (at most the last NS issued)
  if (!ok && tid == 0) {
    for (int r = q_issued - NS < 0 ? 0 : q_issued - NS; r < q_issued; ++r)
      mbar_wait(&full[r % NS], (r / NS) & 1, nullptr);
  }
}

}  // namespace cup
