// Building blocks of the streaming FP64 CG kernel: one-dimensional bulk
// copies (cp.async.bulk, the TMA unit's non-tensor form) of contiguous cell
// windows from global into shared memory, completed on mbarriers, with
// bounded waits.
//
// Alignment: a bulk copy starts on a 16-byte boundary and moves a multiple of
// 16 bytes, so every window is rounded out to even cell indices (compact
// arrays start 256-byte aligned and hold at least one padding cell when the
// cell count is odd, so the rounded-up end stays inside the allocation).
// Copies read this GPU's memory only; no multicast form is used.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cg_common.cuh"
#include "cluster_red.cuh"

namespace eaf {

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One arrival that also announces `bytes` of bulk-copy completions.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of `bar` with the given parity to complete; gives up
// after timeout_ns of global time or when the shared error word is set
// (recording EAF_ETIMEOUT in the first case). Returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          uint64_t timeout_ns) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  uint32_t spins = 0;
  while (!mbar_test(bar, parity)) {
    if ((++spins & 63u) == 0) {
      if (ld_volatile_i32(err) != 0) return false;
      if (global_ns() - t0 > timeout_ns) {
        atomicCAS(err, 0, (int)EAF_ETIMEOUT);
        return false;
      }
    }
  }
  return true;
}
// Bulk copy of `bytes` (a multiple of 16) from global `src` to shared `dst`
// (both 16-byte aligned), completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Orders this thread's generic-proxy global writes before later bulk
// copies (async proxy) that read them, once a barrier has published them.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__host__ __device__ __forceinline__ int even_floor(int v) { return v & ~1; }
__host__ __device__ __forceinline__ int even_ceil(int v) { return (v + 1) & ~1; }

// A window [lo, hi) of cells (even bounds) staged at `buf`.
struct Window {
  const double* buf;
  int lo, hi;
  __device__ __forceinline__ double operator[](int c) const { return buf[c - lo]; }
};

}  // namespace eaf
