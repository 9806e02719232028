// Shared device-side helpers for the sm_100a kernels: bounded mbarrier waits,
// TMA (cp.async.bulk.tensor) loads/stores, 1-D bulk copies and warp/block
// reductions. Nothing here spins without a time limit: every wait gives up
// after kWaitLimitNs, records where in the device error word and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cup {

// Device error word codes (bit flags, OR-ed by any CTA that hits them).
enum : int {
  kDevErrNone = 0,
  kDevErrMbarTimeout = 1,   // an mbarrier wait ran past its time limit
  kDevErrBulkTimeout = 2,   // waiting for a bulk store to drain ran past its limit
  kDevErrNonFinite = 4,     // a reduction saw NaN/Inf
};

constexpr unsigned long long kWaitLimitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Dynamic shared memory rounded up to a 128-byte boundary (TMA destinations
// must be 128-byte aligned); launches reserve 128 extra bytes for this.
__device__ __forceinline__ unsigned char* smem_align128(unsigned char* p) {
  const uint32_t off = smem_u32(p);
  return p + ((128u - (off & 127u)) & 127u);
}

// ---- mbarrier -------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the given phase parity; returns false (and flags the error word)
// if the phase has not completed within kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kWaitLimitNs) {
      if (err) atomicOr(err, kDevErrMbarTimeout);
      return false;
    }
  }
}

// ---- TMA tiled loads / stores (no multicast anywhere in this library) -----
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int c0, int c1, int c2, const void* smem_src) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(smem_src))
      : "memory");
}

// 1-D bulk copy global -> shared (16-B aligned addresses, size multiple of 16).
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// 1-D bulk copy shared -> global.
__device__ __forceinline__ void bulk_store(void* gdst, const void* smem_src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
               "r"(smem_u32(smem_src)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Waits until all committed bulk stores of this thread are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Waits until the shared-memory sources of all but the N most recent committed
// bulk-store groups of this thread have been read (the buffers may be reused).
template <int N_>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N_) : "memory");
}

// Orders this thread's generic-proxy shared-memory writes before subsequent
// async-proxy (TMA / bulk) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- programmatic dependent launch ----------------------------------------
// The step's kernels are launched with programmatic stream serialization: a
// kernel's CTAs may be scheduled while the previous kernel of the stream is
// still finishing (its launch and set-up overlap that kernel's tail). Each
// such kernel calls pdl_wait() before its first access to global memory that
// an earlier kernel writes or reads (everything except the tables written
// once at creation): it returns once the previous kernel has completed and
// its writes are visible. pdl_launch_dependents() then lets the next kernel
// of the stream launch early in turn. Both are no-ops for a kernel launched
// without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_entry() {
  pdl_wait();
  pdl_launch_dependents();
}

// ---- reductions -----------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reduction of NV doubles; result valid in thread 0. `scratch`
// holds at least 32*NV doubles of shared memory.
template <int NV, bool IS_MAX>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = IS_MAX ? warp_max(v[i]) : warp_sum(v[i]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) scratch[i * 32 + wid] = v[i];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = lane < nw ? scratch[i * 32 + lane] : (IS_MAX ? 0.0 : 0.0);
      v[i] = IS_MAX ? warp_max(x) : warp_sum(x);
    }
  }
  __syncthreads();
}

}  // namespace cup
