// Plane-streaming stencil kernels (the device replacement of Cubism's
// BlockLab + Operator::compute block loop, source/operators/Operator.h:112-170).
//
// A CTA owns work items of TY full x-rows by ZC z-planes. For every z plane
// it needs (ZC + 2G planes per item, wrapped periodically in z), one elected
// thread issues TMA tiled loads of NF fields into a ring of NS shared-memory
// plane slots: the TY main rows plus G halo rows below and above (y wraps
// periodically; because y0 is a multiple of TY the halo rows are always a
// contiguous G-row box). The x halo is the periodic wrap of the full row in
// shared memory. Output plane k uses slots for planes k-G..k+G; loads run
// NS-(2G+1) planes ahead of compute. No load ever leaves the tensor bounds,
// so the zero fill of TMA is never used.
#pragma once

#include "common.cuh"

namespace cup {

constexpr int kStreamAcc = 20;

template <int NF>
struct FieldMaps {
  CUtensorMap main[NF];  // box {nx, TY, 1}
  CUtensorMap halo[NF];  // box {nx, G, 1}
};

struct StreamGeom {
  int nx, ny, nz;
  int log2nx;
  int zc;       // z planes per work item
  int items_y;  // ny / TY
  int n_items;  // items_y * nz / zc
};

// Read-only view of the resident planes for the output plane being computed.
template <typename T, int NF, int G, int TY>
struct PlaneCtx {
  static constexpr int ROWS = TY + 2 * G;
  const T* base[2 * G + 1];  // slot base for dz = -G..G
  int nx, mask;
  // value of field f at (x+dx, y+dy, z+dz), y a local row in [0, TY)
  __device__ __forceinline__ T v(int f, int x, int y, int dx, int dy, int dz) const {
    return base[dz + G][(f * ROWS + (G + y + dy)) * nx + ((x + dx) & mask)];
  }
};

template <typename T, int NF, int G, int TY, int NS>
constexpr size_t stream_smem_bytes(int nx) {
  return (size_t)NS * NF * (TY + 2 * G) * nx * sizeof(T) + NS * sizeof(uint64_t) + 32 * kStreamAcc * sizeof(double);
}

// Op must provide:
//   template <class Ctx> __device__ void cell(const Ctx&, int x, int y, int gy, int gz, double* acc) const;
//   __device__ void finish(double* acc, double* scratch) const;  // block epilogue (reductions)
// acc[kStreamAcc] is a per-thread accumulator array, zero-initialised.
template <typename T, int NF, int G, int TY, int NS, class Op>
__global__ void __launch_bounds__(256) k_stencil_stream(const __grid_constant__ FieldMaps<NF> maps,
                                                       const StreamGeom g, Op op, int* err, const int* skip) {
  pdl_entry();
  static_assert(NS >= 2 * G + 1, "ring must hold the stencil planes");
  // a G-row halo box starting at y0 - G (wrapped) stays inside [0, ny) only if y0 is a multiple of TY >= G
  static_assert(TY >= G, "tile height must cover the halo depth");
  if (skip && *skip) return;  // device-side early exit (converged defect correction)
  constexpr int ROWS = TY + 2 * G;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t slot_elems = (size_t)NF * ROWS * nx;
  T* slots = reinterpret_cast<T*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * slot_elems * sizeof(T));
  double* scratch = reinterpret_cast<double*>(full + NS);
  const int tid = threadIdx.x;
  const int PL = g.zc + 2 * G;
  const int my_items = blockIdx.x < g.n_items ? (g.n_items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int L = my_items * PL;
  const uint32_t slot_bytes = (uint32_t)(slot_elems * sizeof(T));

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto issue = [&](int q) {
    const int it = q / PL, j = q - it * PL;
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY;
    int z = zi * g.zc - G + j;
    z = z < 0 ? z + nz : (z >= nz ? z - nz : z);
    const int s = q % NS;
    T* dst = slots + s * slot_elems;
    int ylo = y0 - G;
    if (ylo < 0) ylo += ny;
    int yhi = y0 + TY;
    if (yhi >= ny) yhi -= ny;
    mbar_arrive_expect_tx(&full[s], slot_bytes);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      T* fd = dst + f * ROWS * nx;
      tma_load_3d(fd, &maps.halo[f], 0, ylo, z, &full[s]);
      tma_load_3d(fd + G * nx, &maps.main[f], 0, y0, z, &full[s]);
      tma_load_3d(fd + (G + TY) * nx, &maps.halo[f], 0, yhi, z, &full[s]);
    }
  };

  int q_issued = 0;
  if (tid == 0)
    for (; q_issued < min(L, NS); ++q_issued) issue(q_issued);

  const int cells = nx * TY;
  double acc[kStreamAcc];
#pragma unroll
  for (int i = 0; i < kStreamAcc; ++i) acc[i] = 0.0;
  int a = 0;
  bool ok = true;
  for (int it = 0; it < my_items && ok; ++it) {
    const int item = blockIdx.x + it * gridDim.x;
    const int ty = item % g.items_y, zi = item / g.items_y;
    const int y0 = ty * TY, z0 = zi * g.zc;
    for (int k = 0; k < g.zc; ++k) {
      a = it * PL + k;
      bool mine = true;
#pragma unroll
      for (int d = 0; d <= 2 * G; ++d) mine = mine && mbar_wait(&full[(a + d) % NS], ((a + d) / NS) & 1, err);
      ok = __syncthreads_and(mine);
      if (!ok) break;
      PlaneCtx<T, NF, G, TY> ctx;
#pragma unroll
      for (int d = 0; d <= 2 * G; ++d) ctx.base[d] = slots + ((a + d) % NS) * slot_elems;
      ctx.nx = nx;
      ctx.mask = nx - 1;
      for (int c = tid; c < cells; c += blockDim.x) {
        const int x = c & (nx - 1), y = c >> g.log2nx;
        op.cell(ctx, x, y, y0 + y, z0 + k, acc);
      }
      __syncthreads();
      const int a_next = (k + 1 < g.zc) ? a + 1 : (it + 1) * PL;
      if (tid == 0)
        for (; q_issued < min(L, a_next + NS); ++q_issued) issue(q_issued);
    }
  }
  if (!ok) {
    // Drain the loads this CTA still has in flight (bounded), then leave.
    for (int q = a; q < q_issued; ++q) mbar_wait(&full[q % NS], (q / NS) & 1, nullptr);
    __syncthreads();
    return;
  }
  op.finish(acc, scratch);
}

}  // namespace cup
