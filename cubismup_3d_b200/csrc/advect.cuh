// Advection-diffusion kernels with register z-queues (KernelAdvectDiffuse,
// source/operators/AdvectionDiffusion.cpp:111-144, and the upwind3 + RK2
// stages), the device replacement of Operator::compute's block/lab loop
// (source/operators/Operator.h:112-170) for this operator.
//
// Each thread owns CPT fixed (x, y) columns of a TY x nx row tile and marches
// down z. Planes arrive by TMA into a ring of NS shared-memory slots (TY main
// rows plus G periodic halo rows per field; the x halo is the row's periodic
// wrap). When plane j lands, a thread
//   1. pushes its columns' centre values into a register queue of the last
//      2G+1 planes (the z stencil),
//   2. finishes output plane j-2G: adds the z terms (from the queue) to the
//      x/y partial it computed G planes earlier, and stores it,
//   3. computes the x/y partial of plane j (x/y neighbours from shared memory,
//      advecting velocity from the queue),
// and the slot is released at once: only planes in flight occupy shared
// memory, so NS-1 planes of loads are always outstanding. For RK2 stage 2 the
// point-wise base rows u^n of the output plane ride in the same slot as the
// load that completes it. Work items (TY rows x ZC planes) of a CTA form one
// flat load stream, so the pipeline never drains between items.
#pragma once

#include "common.cuh"
#include "ops.cuh"
#include "stencil.cuh"

namespace cup {

struct AdvectMaps {
  CUtensorMap main[3];  // stencil fields, box {nx, TY, 1}
  CUtensorMap halo[3];  // stencil fields, box {nx, G, 1}
  CUtensorMap base[3];  // stage-2 point-wise fields, box {nx, TY, 1}
};

// SCHEME 0: central2 (reference) Euler; 1: upwind3 stage 1; 2: upwind3 stage 2.
template <int SCHEME>
struct AdvectTraits {
  static constexpr int G = SCHEME == 0 ? 1 : 2;
  static constexpr bool BASE = SCHEME == 2;
};

template <typename T, int SCHEME, int TY, int NS, int CPT>
constexpr size_t advect_smem_bytes(int nx) {
  constexpr int G = AdvectTraits<SCHEME>::G;
  return (size_t)NS * (3 * (TY + 2 * G) + (AdvectTraits<SCHEME>::BASE ? 3 * TY : 0)) * nx * sizeof(T) +
         NS * sizeof(uint64_t);
}

// blockDim.x * CPT must equal TY * nx (<= 512 threads).
// NXC, ZCC: nx and the planes per work item fixed at compile time (0: read
// from g); fixed, the stencil's shared-memory offsets are immediates and the
// ring slot of each plane is known when NS divides the item's plane count.
template <typename T, int SCHEME, int TY, int NS, int CPT, int NXC = 0, int ZCC = 0>
__global__ void __launch_bounds__(512) k_advect_zq(const __grid_constant__ AdvectMaps maps, const StreamGeom g,
                                                  T* __restrict__ ou, T* __restrict__ ov, T* __restrict__ ow, DtArg dt,
                                                  double h, double nu, double ux, double uy, double uz, int* err) {
  pdl_entry();
  constexpr int G = AdvectTraits<SCHEME>::G;
  constexpr bool BASE = AdvectTraits<SCHEME>::BASE;
  constexpr int ROWS = TY + 2 * G;
  constexpr int Q = 2 * G + 1;
  // a G-row halo box starting at y0 - G (wrapped) stays inside [0, ny) only if y0 is a multiple of TY >= G
  static_assert(TY >= G, "tile height must cover the halo depth");
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  const int nx = NXC ? NXC : g.nx, ny = g.ny, nz = g.nz;
  const int zc = ZCC ? ZCC : g.zc;
  const size_t field_elems = (size_t)ROWS * nx;
  const size_t stencil_elems = 3 * field_elems;
  const size_t slot_elems = stencil_elems + (BASE ? (size_t)3 * TY * nx : 0);
  T* slots = reinterpret_cast<T*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * slot_elems * sizeof(T));
  const int tid = threadIdx.x;
  const int PL = zc + 2 * G;
  const int my_items = blockIdx.x < g.n_items ? (g.n_items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int L = my_items * PL;
  const uint32_t stencil_bytes = (uint32_t)(stencil_elems * sizeof(T));
  const uint32_t base_bytes = (uint32_t)(3 * TY * nx * sizeof(T));

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
    T* dst = slots + s * slot_elems;
    int ylo = y0 - G;
    if (ylo < 0) ylo += ny;
    int yhi = y0 + TY;
    if (yhi >= ny) yhi -= ny;
    const bool with_base = BASE && j >= 2 * G;
    mbar_arrive_expect_tx(&full[s], stencil_bytes + (with_base ? base_bytes : 0u));
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      T* fd = dst + f * field_elems;
      tma_load_3d(fd, &maps.halo[f], 0, ylo, z, &full[s]);
      tma_load_3d(fd + G * nx, &maps.main[f], 0, y0, z, &full[s]);
      tma_load_3d(fd + (G + TY) * nx, &maps.halo[f], 0, yhi, z, &full[s]);
    }
    if (with_base) {
      const int zk = z0 + (j - 2 * G);  // output plane completed by this load (< nz)
#pragma unroll
      for (int f = 0; f < 3; ++f) tma_load_3d(dst + stencil_elems + f * TY * nx, &maps.base[f], 0, y0, zk, &full[s]);
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
    cy[i] = NXC ? c / NXC : c >> g.log2nx;
  }
  const double dtv = dt.get();
  const T facA = (T)(SCHEME == 0 ? -dtv / (2 * h) : -dtv / (6 * h));
  const T facD = (T)((nu / h) * (dtv / h));
  const T uinf[3] = {(T)ux, (T)uy, (T)uz};

  // Register rings: qv holds the centre values of the last Q = 2G+1 planes
  // (plane j in slot j % Q), part the x/y partials awaiting their z terms
  // (the partial of load j in slot j % G). The plane loop is unrolled by
  // U = lcm(Q, G) and every item's PL = ZC + 2G planes is a multiple of U, so
  // all ring indices fold to constants: no register shuffling.
  constexpr int U = ZCC ? ZCC + 2 * G : ((G == 1) ? 3 : 10);
  constexpr bool SLOT_CT = ZCC != 0 && (ZCC + 2 * G) % NS == 0;  // ring slot of plane j is j % NS
  static_assert(ZCC % 2 == 0, "paired barriers need an even plane count");
  T qv[3][Q][CPT];
  T part[3][G][CPT];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int d = 0; d < Q; ++d)
#pragma unroll
      for (int i = 0; i < CPT; ++i) qv[f][d][i] = (T)0;
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int d = 0; d < G; ++d)
#pragma unroll
      for (int i = 0; i < CPT; ++i) part[f][d][i] = (T)0;

  // One block barrier per plane (slot release). Each thread waits on the
  // slot's mbarrier itself; a thread whose wait timed out stops waiting and
  // computing but keeps taking the barrier, so the block never deadlocks and
  // the error word tells the host.
  bool ok = true;
  int q = 0;
  for (int it = 0; it < my_items; ++it) {
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY, z0 = zi * zc;
    const int q0 = q;  // first load of the item (a multiple of NS when SLOT_CT)
    for (int j0 = 0; j0 < PL; j0 += U) {
#pragma unroll
      for (int jj = 0; jj < U; ++jj) {
        const int j = j0 + jj;
        const int s = SLOT_CT ? jj % NS : q % NS;
        const uint32_t phase = SLOT_CT ? ((q0 / NS + jj / NS) & 1) : ((q / NS) & 1);
        if (ok) ok = mbar_wait(&full[s], phase, err);
        if (ok) {
          const T* sl = slots + s * slot_elems;
          const int QN = jj % Q;  // slot of the newest plane
          // 1. centre values of plane j
#pragma unroll
          for (int f = 0; f < 3; ++f)
#pragma unroll
            for (int i = 0; i < CPT; ++i) qv[f][QN][i] = sl[f * field_elems + (G + cy[i]) * nx + cx[i]];
          // 2. finish output plane k = j - 2G (queue slot of plane k + d - G: (jj - 2G + d) mod Q)
          if (j >= 2 * G) {
            const int k = j - 2 * G;
            const int QC = (jj + 3 * Q - G) % Q;       // centre (load j - G)
            const int QM1 = (jj + 3 * Q - G - 1) % Q;  // plane k - 1
            const int QP1 = (jj + 3 * Q - G + 1) % Q;  // plane k + 1
            const int QM2 = (jj + 3 * Q - G - 2) % Q;  // plane k - 2 (G = 2)
            const int QP2 = (jj + 3 * Q - G + 2) % Q;  // plane k + 2 (G = 2)
            const int PS = jj % G;                      // partial of load j - G
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
              const size_t o = gidx(cx[i], y0 + cy[i], z0 + k, nx, ny);
              const T ww = qv[2][QC][i] + uinf[2];
              T outv[3];
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const T f0 = qv[f][QC][i];
                T dz;
                if constexpr (SCHEME == 0) {
                  dz = qv[f][QP1][i] - qv[f][QM1][i];
                } else {
                  dz = up3(ww, qv[f][QM2][i], qv[f][QM1][i], f0, qv[f][QP1][i], qv[f][QP2][i]);
                }
                const T lz = qv[f][QM1][i] + qv[f][QP1][i];
                outv[f] = f0 + part[f][PS][i] + facA * (ww * dz) + facD * (lz - f0 * 6);
              }
              if constexpr (BASE) {
                const T* bs = sl + stencil_elems + cy[i] * nx + cx[i];
                ou[o] = (T)0.5 * (bs[0] + outv[0]);
                ov[o] = (T)0.5 * (bs[TY * nx] + outv[1]);
                ow[o] = (T)0.5 * (bs[2 * TY * nx] + outv[2]);
              } else {
                ou[o] = outv[0];
                ov[o] = outv[1];
                ow[o] = outv[2];
              }
            }
          }
          // 3. x/y partial of plane j (output plane j - G), into slot j % G
          if (j >= G && j < G + zc) {
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
              const T uu = qv[0][QN][i] + uinf[0], vv = qv[1][QN][i] + uinf[1];
              const int x = cx[i], r = G + cy[i];
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const T* F = sl + f * field_elems;
                const T f0 = qv[f][QN][i];
                const T xm1 = F[r * nx + ((x - 1) & mask)], xp1 = F[r * nx + ((x + 1) & mask)];
                const T ym1 = F[(r - 1) * nx + x], yp1 = F[(r + 1) * nx + x];
                T dx, dy;
                if constexpr (SCHEME == 0) {
                  dx = xp1 - xm1;
                  dy = yp1 - ym1;
                } else {
                  const T xm2 = F[r * nx + ((x - 2) & mask)], xp2 = F[r * nx + ((x + 2) & mask)];
                  const T ym2 = F[(r - 2) * nx + x], yp2 = F[(r + 2) * nx + x];
                  dx = up3(uu, xm2, xm1, f0, xp1, xp2);
                  dy = up3(vv, ym2, ym1, f0, yp1, yp2);
                }
                part[f][PS][i] = facA * (uu * dx + vv * dy) + facD * (yp1 + ym1 + xp1 + xm1);
              }
            }
          }
        }
        // rings of 4+ slots: one block barrier per two planes (slots of loads
        // q-1 and q fully consumed, refill both; PL is even, so a pair never
        // straddles items); shallower rings keep one barrier per plane
        if constexpr (NS >= 4) {
          if (q & 1) {
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
  if (!ok && tid == 0) {
    // bounded drain of this CTA's loads still in flight (at most the last NS issued)
    for (int r = q_issued - NS < 0 ? 0 : q_issued - NS; r < q_issued; ++r)
      mbar_wait(&full[r % NS], (r / NS) & 1, nullptr);
  }
}

}  // namespace cup
