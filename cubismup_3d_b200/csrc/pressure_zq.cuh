// Pressure-stage kernels of the FP32 defect-correction step, register z-queue
// form; every pass recomputes b = KernelPressureRHS(u*)
// (source/operators/PressureRHS.cpp:51-76) from u* (div_xy / div_b:
// bit-identical in each):
//   RHS_RES    the first FP64 residual r = b - h/4 L_2h p of the warm start,
//              r in FP32 for the FFT solve.
//   RES        r = b - h/4 L_2h p before a further correction solve, minus the
//              class means of b (its null-mode part), in FP32.
//   GRAD_CHECK KernelGradP (source/operators/PressureProjection.cpp:38-50) on
//              u* with the current p, written to a separate buffer so that it
//              can be redone, fused with the residual check of that p (the
//              divergence left by the projection is this residual) and, on
//              the first check of a step, with the warm start of the next
//              step's solve: the linear extrapolation 2 p_{n+1} - p_n. (The
//              unpredictable part of b is the white FP32 rounding noise of the
//              stored velocity; a quadratic extrapolation amplifies it more
//              than it gains on the smooth part.)
//   GRAD_CHECK_BOX  GRAD_CHECK with an obstacle: the max |u + uinf| leaves
//              out the obstacle's box (the penalization pass covers it).
// BD: with the obstacle, b also carries the RHS obstacle terms
// (PressureRHS.cpp:78-112, 215-256), formed on the obstacle's box by one small
// pass and added back here on the box.
// L_2h is the wide-stencil Laplacian (neighbours at +-2) the spectral solve
// inverts; p is FP64 throughout.
//
// Structure as k_advect_zq: each thread owns CPT (x, y) columns of a TY x nx
// row tile and marches down z; planes of p (TY + 4 rows: the +-2 halo in y)
// arrive by TMA into a ring of NS slots, the centre values of the last 5
// planes sit in a register queue (the z stencil), the x/y part of each plane
// is computed on arrival and completed two planes later. The point-wise fields
// of an output plane (u*, the previous p) ride in the slot of the load that
// completes it.
// Partial sums per CTA: the 18-value residual layout (sum r^2 with the null
// parts removed after check 0, sum b^2 and the class sums of r at check 0,
// class sums of p); GRAD_CHECK then adds max |u + uinf| and the kinetic
// energy: 20 per CTA.
#pragma once

#include "common.cuh"
#include "ops.cuh"
#include "stencil.cuh"

namespace cup {

enum { PZQ_RHS_RES = 0, PZQ_RES = 1, PZQ_GRAD_CHECK = 2, PZQ_GRAD_CHECK_BOX = 3 };

template <int MODE>
constexpr bool pzq_grad() {
  return MODE == PZQ_GRAD_CHECK || MODE == PZQ_GRAD_CHECK_BOX;
}

struct PzqMaps {
  CUtensorMap p_main, p_halo;  // FP64 p: box {nx, TY, 1} and {nx, 2, 1}
  CUtensorMap f_main[3];       // u*, v*, w* (storage type): box {nx, TY, 1}
  CUtensorMap v_halo;          // v*: box {nx, 1, 1}
  CUtensorMap h_main;          // FP64 pressure of the previous step p_n: box {nx, TY, 1} (GRAD_CHECK)
};

// Values per CTA in the partial-sum buffer.
template <int MODE>
constexpr int pzq_partials_per_cta() {
  return pzq_grad<MODE>() ? 20 : 18;
}

struct PzqParams {
  DtArg dt;
  double h;
  double uinf[3];
  // GRAD_CHECK: extrapolation order of the next step's warm start from the
  // current p and the previous step's p_n (0: p, 1: 2 p - p_n; negative: the
  // warm start is not written)
  int pred_order;
  double* pred_out;
  Box box;  // GRAD_CHECK_BOX: the obstacle's box
  // BD: the obstacle terms of the RHS on the box (b2 - b0, box [z][y][x]
  // order), added to the b the pass recomputes from u*
  const double* bdelta;
};

// Byte layout of one ring slot (all parts multiples of 64 B for nx >= 16).
template <typename T, int MODE, int TY>
struct PzqSlot {
  static constexpr int G = 2;
  __host__ __device__ static size_t p_bytes(int nx) { return (size_t)(TY + 2 * G) * nx * sizeof(double); }
  // b from u*: u [TY], v [TY + 2], w [TY] rows of T
  __host__ __device__ static size_t u_off(int nx) { return p_bytes(nx); }
  __host__ __device__ static size_t v_off(int nx) { return u_off(nx) + (size_t)TY * nx * sizeof(T); }
  __host__ __device__ static size_t w_off(int nx) { return v_off(nx) + (size_t)(TY + 2) * nx * sizeof(T); }
  __host__ __device__ static size_t div_end(int nx) { return w_off(nx) + (size_t)TY * nx * sizeof(T); }
  // GRAD_CHECK: u*, v*, w* [TY] rows of T of the output plane
  __host__ __device__ static size_t f_off(int nx, int f) { return div_end(nx) + (size_t)f * TY * nx * sizeof(T); }
  // GRAD_CHECK: then the rows of the previous step's p [TY] of double
  __host__ __device__ static size_t h_off(int nx) { return f_off(nx, 3); }
  __host__ __device__ static size_t bytes(int nx) {
    size_t s = pzq_grad<MODE>() ? h_off(nx) + (size_t)TY * nx * sizeof(double) : div_end(nx);
    return (s + 127) / 128 * 128;
  }
};

template <typename T, int MODE, int TY, int NS>
constexpr size_t pzq_smem_bytes_host(int nx) {
  return (size_t)NS * PzqSlot<T, MODE, TY>::bytes(nx) + NS * sizeof(uint64_t) + 18 * 32 * sizeof(double);
}

// blockDim.x * CPT == TY * nx (<= 512 threads), TY even.
// NXC, ZCC: nx and the planes per work item fixed at compile time (0: read
// from g); fixed, the stencil's shared-memory offsets are immediates and the
// ring slot of each plane is known.
// BD: the obstacle terms of b added back on the box (prm.bdelta).
template <typename T, int MODE, int TY, int NS, int CPT, int NXC = 0, int ZCC = 0, bool BD = false>
__global__ void __launch_bounds__(512) k_pres_zq(const __grid_constant__ PzqMaps maps, const StreamGeom g,
                                                T* __restrict__ ou, T* __restrict__ ov, T* __restrict__ ow,
                                                float* __restrict__ rout,
                                                double* __restrict__ partials, const double* __restrict__ rmean,
                                                const PzqParams prm, int* err, const int* skip) {
  pdl_entry();
  constexpr int G = 2;
  constexpr int Q = 2 * G + 1;
  constexpr int U = ZCC ? ZCC + 2 * G : 10;  // planes per unrolled chunk: a whole item, or lcm(Q, G)
  constexpr bool SLOT_CT = ZCC != 0 && (ZCC + 2 * G) % NS == 0;  // ring slot of plane j is j % NS
  static_assert(TY >= G && TY % 2 == 0, "tile height must cover the halo depth and keep the row parity");
  static_assert(ZCC % 2 == 0, "paired barriers and the z parity need an even plane count");
  using Slot = PzqSlot<T, MODE, TY>;
  static_assert(BD || MODE != PZQ_GRAD_CHECK_BOX, "with the obstacle, b needs its terms");
  if (skip && *skip) return;  // converged defect correction: nothing to check
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  const int nx = NXC ? NXC : g.nx, ny = g.ny, nz = g.nz;
  const int zc = ZCC ? ZCC : g.zc;
  const size_t slot_bytes = Slot::bytes(nx);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * slot_bytes);
  double* scratch = reinterpret_cast<double*>(full + NS);
  const int tid = threadIdx.x;
  const int PL = zc + 2 * G;
  const int my_items = blockIdx.x < g.n_items ? (g.n_items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int L = my_items * PL;
  const uint32_t p_bytes = (uint32_t)Slot::p_bytes(nx);
  const uint32_t rowsT = (uint32_t)(TY * nx * sizeof(T));
  const uint32_t rowsD = (uint32_t)(TY * nx * sizeof(double));

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
    unsigned char* dst = smem_raw + s * slot_bytes;
    int ylo = y0 - G;
    if (ylo < 0) ylo += ny;
    int yhi = y0 + TY;
    if (yhi >= ny) yhi -= ny;
    uint32_t bytes = p_bytes;
    const bool xy_plane = j >= G && j < G + zc;    // planes whose x/y part is computed
    const bool w_plane = j >= 1 && j < PL - 1;        // planes at z0-1 .. z0+zc (w at z +- 1)
    const bool out_plane = j >= 2 * G;                // completes output plane j - 2G
    if (xy_plane) bytes += rowsT + (uint32_t)((TY + 2) * nx * sizeof(T));
    if (w_plane) bytes += rowsT;
    if constexpr (pzq_grad<MODE>()) {
      if (out_plane) bytes += 3 * rowsT + (prm.pred_order >= 1 ? rowsD : 0u);
    }
    mbar_arrive_expect_tx(&full[s], bytes);
    double* P = reinterpret_cast<double*>(dst);
    tma_load_3d(P, &maps.p_halo, 0, ylo, z, &full[s]);
    tma_load_3d(P + G * nx, &maps.p_main, 0, y0, z, &full[s]);
    tma_load_3d(P + (G + TY) * nx, &maps.p_halo, 0, yhi, z, &full[s]);
    if (xy_plane) {
      tma_load_3d(dst + Slot::u_off(nx), &maps.f_main[0], 0, y0, z, &full[s]);
      T* V = reinterpret_cast<T*>(dst + Slot::v_off(nx));
      tma_load_3d(V, &maps.v_halo, 0, y0 == 0 ? ny - 1 : y0 - 1, z, &full[s]);
      tma_load_3d(V + nx, &maps.f_main[1], 0, y0, z, &full[s]);
      tma_load_3d(V + (TY + 1) * nx, &maps.v_halo, 0, yhi, z, &full[s]);
    }
    if (w_plane) tma_load_3d(dst + Slot::w_off(nx), &maps.f_main[2], 0, y0, z, &full[s]);
    if (out_plane) {
      const int zk = z0 + (j - 2 * G);  // output plane completed by this load (< nz)
      if constexpr (pzq_grad<MODE>()) {
#pragma unroll
        for (int f = 0; f < 3; ++f) tma_load_3d(dst + Slot::f_off(nx, f), &maps.f_main[f], 0, y0, zk, &full[s]);
        if (prm.pred_order >= 1) tma_load_3d(dst + Slot::h_off(nx), &maps.h_main, 0, y0, zk, &full[s]);
      }
    }
  };

  int q_issued = 0;
  if (tid == 0)
    for (; q_issued < min(L, NS); ++q_issued) issue(q_issued);

  const int mask = nx - 1;
  // per column: its cell, the shared-memory offsets of its x/y neighbours in
  // a slot, and (after check 0) the class means of b at both z parities
  int cx[CPT], cy[CPT];
  int xm1[CPT], xp1[CPT], xm2[CPT], xp2[CPT];
  double rm[CPT][2];
#pragma unroll
  for (int i = 0; i < CPT; ++i) {
    const int c = tid + i * blockDim.x;
    cx[i] = c & mask;
    cy[i] = NXC ? c / NXC : c >> g.log2nx;
    xm1[i] = (cx[i] - 1) & mask;
    xp1[i] = (cx[i] + 1) & mask;
    xm2[i] = (cx[i] - 2) & mask;
    xp2[i] = (cx[i] + 2) & mask;
#pragma unroll
    for (int zp = 0; zp < 2; ++zp)
      rm[i][zp] = MODE == PZQ_RHS_RES ? 0.0 : rmean[(cx[i] & 1) | ((cy[i] & 1) << 1) | (zp << 2)];
  }
  const size_t plane = (size_t)nx * ny;
  const double dtv = prm.dt.get();
  const double h = prm.h;
  const double cL = 0.25 * h;           // h^3 / (4 h^2)
  const double facB = 0.5 * h * h / dtv;  // KernelPressureRHS scaling
  const double facG = -0.5 * dtv / h;     // KernelGradP scaling

  double pq[Q][CPT];
  T wq[Q][CPT];
  // x/y parts of the planes in flight (G of them): Laplacian, divergence and
  // (GRAD_CHECK) the gradient of p and the u*, v* centre values
  double partL[G][CPT];
  T partD[G][CPT];               // x/y part of the divergence (b from u*: div_xy, div_b)
  double partB[BD ? G : 1][CPT];  // BD: the obstacle terms of the output cell, loaded two planes ahead
  double gA[G][CPT], gB[G][CPT];  // x- and y-gradient of p (GRAD_CHECK)
  double pc[CPT][2], rc[CPT][2];  // parity-class sums of p and r by z parity
  double acc0 = 0, acc1 = 0;
  // extremes of each corrected velocity component: max |u + uinf| over the
  // cells is max(|umax + uinf|, |umin + uinf|), so the FP64 max needs no
  // per-cell conversion
  T vmax[3], vmin[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    vmax[c] = (T)-INFINITY;
    vmin[c] = (T)INFINITY;
  }
#pragma unroll
  for (int d = 0; d < Q; ++d)
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
      pq[d][i] = 0.0;
      wq[d][i] = (T)0;
    }
#pragma unroll
  for (int d = 0; d < G; ++d)
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
      partL[d][i] = gA[d][i] = gB[d][i] = 0.0;
      partD[d][i] = (T)0;
      if constexpr (BD) partB[d][i] = 0.0;
    }
#pragma unroll
  for (int i = 0; i < CPT; ++i) pc[i][0] = pc[i][1] = rc[i][0] = rc[i][1] = 0.0;

  bool ok = true;
  int q = 0;
  for (int it = 0; it < my_items; ++it) {
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY, z0 = zi * zc;
    size_t obase[CPT];  // output index of plane z0
#pragma unroll
    for (int i = 0; i < CPT; ++i) obase[i] = gidx(cx[i], y0 + cy[i], z0, nx, ny);
    const int q0 = q;  // first load of the item (a multiple of NS when SLOT_CT)
    for (int j0 = 0; j0 < PL; j0 += U) {
#pragma unroll
      for (int jj = 0; jj < U; ++jj) {
        const int j = j0 + jj;
        if (j >= PL) break;  // items of PL planes, PL not a multiple of U
        const int s = SLOT_CT ? jj % NS : q % NS;
        const uint32_t phase = SLOT_CT ? ((q0 / NS + jj / NS) & 1) : ((q / NS) & 1);
        if (ok) ok = mbar_wait(&full[s], phase, err);
        if (ok) {
          const unsigned char* sl = smem_raw + s * slot_bytes;
          const double* P = reinterpret_cast<const double*>(sl);
          const int QN = jj % Q;
#pragma unroll
          for (int i = 0; i < CPT; ++i) pq[QN][i] = P[(G + cy[i]) * nx + cx[i]];
          if (j >= 1 && j < PL - 1) {
            const T* W = reinterpret_cast<const T*>(sl + Slot::w_off(nx));
#pragma unroll
            for (int i = 0; i < CPT; ++i) wq[QN][i] = W[cy[i] * nx + cx[i]];
          }
          // output plane k = j - 2G (z parity of k = jj parity: z0 and j0 are even)
          if (j >= 2 * G) {
            const int k = j - 2 * G;
            const int QC = (jj + 3 * Q - G) % Q;
            const int QM1 = (jj + 3 * Q - G - 1) % Q, QP1 = (jj + 3 * Q - G + 1) % Q;
            const int QM2 = (jj + 3 * Q - G - 2) % Q, QP2 = (jj + 3 * Q - G + 2) % Q;
            const int PS = jj % G;
            const int zp = jj & 1;
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
              const size_t o = obase[i] + (size_t)k * plane;
              const int c = cy[i] * nx + cx[i];
              const double p0 = pq[QC][i];
              const double lap = partL[PS][i] + (pq[QP2][i] + pq[QM2][i] - 2 * p0);
              pc[i][zp] += p0;
              // b from u* (x/y part on arrival, z part here), plus the obstacle terms on the box
              double b = div_b<T>(facB, partD[PS][i], wq[QP1][i], wq[QM1][i]);
              if constexpr (BD) b += partB[PS][i];
              if constexpr (MODE == PZQ_RHS_RES) {
                const double r = b - cL * lap;
                rc[i][zp] += r;  // the class means of b (only check 0 needs them)
                rout[o] = (float)r;
                acc0 += r * r;
                acc1 += b * b;
              } else {
                const double r = b - cL * lap;
                const double rp = r - rm[i][zp];
                acc0 += rp * rp;
                if constexpr (MODE == PZQ_RES) {
                  rout[o] = (float)rp;
                } else {
                  // the FP64 correction rounded once to the storage type, then added
                  const T tu = reinterpret_cast<const T*>(sl + Slot::f_off(nx, 0))[c] + (T)(facG * gA[PS][i]);
                  const T tv = reinterpret_cast<const T*>(sl + Slot::f_off(nx, 1))[c] + (T)(facG * gB[PS][i]);
                  const T tw = reinterpret_cast<const T*>(sl + Slot::f_off(nx, 2))[c] +
                               (T)(facG * (pq[QP1][i] - pq[QM1][i]));
                  ou[o] = tu;
                  ov[o] = tv;
                  ow[o] = tw;
                  // warm start of the next step: linear extrapolation in the step index
                  if (prm.pred_order >= 0) {
                    const double* Hn = reinterpret_cast<const double*>(sl + Slot::h_off(nx));
                    prm.pred_out[o] = prm.pred_order == 1 ? 2 * p0 - Hn[c] : p0;
                  }
                  if (MODE != PZQ_GRAD_CHECK_BOX || !prm.box.contains(cx[i], y0 + cy[i], z0 + k, nx, ny, nz)) {
                    vmax[0] = fmax(vmax[0], tu);
                    vmin[0] = fmin(vmin[0], tu);
                    vmax[1] = fmax(vmax[1], tv);
                    vmin[1] = fmin(vmin[1], tv);
                    vmax[2] = fmax(vmax[2], tw);
                    vmin[2] = fmin(vmin[2], tw);
                  }
                  // kinetic energy |u|^2/2: squares in the storage type, FP64 sum
                  acc1 += 0.5 * (double)(tu * tu + tv * tv + tw * tw);
                }
              }
            }
          }
          // x/y part of plane j (output plane j - G)
          if (j >= G && j < G + zc) {
            const int PS = jj % G;
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
              const int x = cx[i];
              const double p0 = pq[QN][i];
              const double* Pc = P + (G + cy[i]) * nx;  // this column's row of p
              partL[PS][i] = (Pc[xp2[i]] + Pc[xm2[i]] - 2 * p0) + (Pc[2 * nx + x] + Pc[x - 2 * nx] - 2 * p0);
              {
                const T* Urow = reinterpret_cast<const T*>(sl + Slot::u_off(nx)) + cy[i] * nx;
                const T* Vc = reinterpret_cast<const T*>(sl + Slot::v_off(nx)) + (cy[i] + 1) * nx;  // row of v*
                partD[PS][i] = div_xy<T>(Urow[xp1[i]], Urow[xm1[i]], Vc[nx + x], Vc[x - nx]);
              }
              if constexpr (BD) {
                // the box's b2 - b0 of output cell (x, y, z0 + j - G), used two planes later
                const int bi = prm.box.index(x, y0 + cy[i], z0 + j - G, nx, ny, nz);
                partB[PS][i] = bi >= 0 ? __ldg(prm.bdelta + bi) : 0.0;
              }
              if constexpr (pzq_grad<MODE>()) {
                gA[PS][i] = Pc[xp1[i]] - Pc[xm1[i]];
                gB[PS][i] = Pc[nx + x] - Pc[x - nx];
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
  // per-CTA partial sums
  {
    constexpr int NPV = pzq_partials_per_cta<MODE>();
    double v[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) v[k] = 0.0;
    v[0] = acc0;
    v[1] = pzq_grad<MODE>() ? 0.0 : acc1;
#pragma unroll
    for (int i = 0; i < CPT; ++i)
#pragma unroll
      for (int zp = 0; zp < 2; ++zp) {
        const int cls = (cx[i] & 1) | ((cy[i] & 1) << 1) | (zp << 2);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          v[2 + c] += c == cls ? pc[i][zp] : 0.0;
          v[10 + c] += c == cls ? rc[i][zp] : 0.0;
        }
      }
    block_reduce<18, false>(v, scratch);
    if constexpr (pzq_grad<MODE>()) {
      double accM = 0.0;
      if (vmax[0] >= vmin[0]) {  // this thread corrected at least one cell
#pragma unroll
        for (int c = 0; c < 3; ++c)
          accM = fmax(accM, fmax(fabs((double)vmax[c] + prm.uinf[c]), fabs((double)vmin[c] + prm.uinf[c])));
      }
      double mx[1] = {accM};
      double ke[1] = {acc1};
      block_reduce<1, true>(mx, scratch);
      block_reduce<1, false>(ke, scratch + 32);
      if (tid == 0) {
        partials[NPV * blockIdx.x + 18] = mx[0];
        partials[NPV * blockIdx.x + 19] = ke[0];
      }
    }
    if (tid == 0)
      for (int k = 0; k < 18; ++k) partials[NPV * blockIdx.x + k] = v[k];
  }
}

}  // namespace cup
