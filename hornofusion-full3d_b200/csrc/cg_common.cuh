// Device building blocks shared by the pressure-CG kernels: mesh indexing in
// the compact device layout, bounded-wait group barriers and deterministic
// block/group reductions.
//
// Compact device layout (one system): interior cells only, flat index
//   c = i + nr*(j + nth*k),  0 <= i < nr, 0 <= j < nth, 0 <= k < nz,
// r fastest (the reference's column-major order without the halo ring).
// theta neighbours wrap (src/mod_mpi_topology.f90:303-311); r and z
// neighbours outside the mesh read as zero, which is what the reference's
// Krylov vectors hold in their r/z halos (src/mod_solver_3d.f90:505-507,526).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "eafcg.h"

namespace eaf {

constexpr double kSmall = 1.0e-30;  // SMALL, src/mod_constants.f90:53

// Unsigned division by a runtime divisor d >= 1 for numerators below 2^31:
// q = (umulhi(n, m) + n) >> s with s = ceil(log2 d) and
// m = floor(2^32 (2^s - d) / d) + 1 (the round-up multiplier method of
// Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994).
struct FastDiv {
  uint32_t d, m, s;
  __host__ __device__ FastDiv() : d(1), m(1), s(0) {}
  __host__ __device__ explicit FastDiv(uint32_t div) : d(div) {
    s = 0;
    while ((1ull << s) < d) ++s;
    m = (uint32_t)(((1ull << 32) * ((1ull << s) - d)) / d + 1);
  }
  __device__ __forceinline__ uint32_t div(uint32_t n) const {
    return (__umulhi(n, m) + n) >> s;
  }
};

struct MeshDims {
  int nr, nth, nz;
  int n;       // nr*nth*nz
  int plane;   // nr*nth
  FastDiv fd_nr, fd_nth;
};

__device__ __forceinline__ void cell_ijk(const MeshDims& d, int c, int& i, int& j,
                                         int& k) {
  uint32_t t = d.fd_nr.div((uint32_t)c);
  i = c - (int)t * d.nr;
  uint32_t kk = d.fd_nth.div(t);
  j = (int)t - (int)kk * d.nth;
  k = (int)kk;
}

// ---------------------------------------------------------------------------
// Memory-model helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long* p,
                                                    unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) {
  return *(const volatile int*)p;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------------------
// Group barrier: `nb` co-resident blocks (a cooperative launch, or one lane
// of a batched launch) meet on a 64-bit arrival counter that is zeroed
// before the launch. Every wait is bounded by `timeout_ns` of global time;
// on expiry the waiter records EAF_ETIMEOUT in the shared error word and all
// waiters of the group leave. A group of one block only needs __syncthreads.
// ---------------------------------------------------------------------------
// Largest group of a persistent launch (blocks) and most sums reduced at
// once; the launchers never exceed them.
constexpr int kMaxGroupBlocks = 1184;
constexpr int kMaxGroupSlots = 3;

struct Group {
  unsigned long long* counter;
  int* err;
  double* part;       // [slots][nb] block partials of this group
  double* stage;      // shared memory for kMaxGroupSlots * nb partials
  int nb;             // blocks in the group
  int bid;            // this block's index in the group
  uint64_t timeout_ns;
  unsigned long long epoch;  // barriers passed (meaningful in thread 0)
  int pq_seq = 0;            // release-free p.q all-reduces passed (all threads)
};

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

// Memory-ordering forms of the group barrier (all correct under the PTX
// memory model; they differ in cost):
//   0  full fences around a release add, acquire polls;
//   1  release add after the CTA barrier, acquire polls, no extra fences
//      (bar.sync orders the block's writes before thread 0's release, and
//      the acquire that observes the last arrival orders what follows);
//   2  release add, relaxed polls, one acquire fence after the last poll.
constexpr int kBarrierForm = 1;
// Form of group_allsum: 0-2 as above (full block barriers around the group
// barrier), 3 the warp-0 form with split block barriers (group_allsum_w0).
#ifndef EAF_ALLSUM_FORM
#define EAF_ALLSUM_FORM 3
#endif
constexpr int kAllsumForm = EAF_ALLSUM_FORM;

template <int FORM = kBarrierForm>
__device__ __forceinline__ bool group_barrier(Group& g) {
  __shared__ int s_ok;
  if (g.nb == 1) {
    __syncthreads();
    return true;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    g.epoch += 1;
    const unsigned long long target = g.epoch * (unsigned long long)g.nb;
    if (FORM == 0) __threadfence();
    red_release_add_u64(g.counter, 1ull);
    int ok = 1;
    uint64_t t0 = 0;
    uint32_t spins = 0;
    while ((FORM == 2 ? ld_relaxed_u64(g.counter) : ld_acquire_u64(g.counter)) < target) {
      if ((++spins & 63u) == 0) {
        if (spins == 64u) t0 = global_ns();
        if (ld_volatile_i32(g.err) != 0) { ok = 0; break; }
        if (global_ns() - t0 > g.timeout_ns) {
          atomicCAS(g.err, 0, (int)EAF_ETIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    if (FORM == 0) __threadfence();
    if (FORM == 2) fence_acq_rel_gpu();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// Deterministic reductions. The warp stage is an xor butterfly, the block
// stage folds warp partials in warp order, and the group stage has warp 0 of
// every block fold the `nb` block partials in the same fixed order, so every
// block of the group obtains the bit-identical total (the exit tests and
// step lengths of all blocks therefore agree).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_allsum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int NV, typename T>
__device__ __forceinline__ void block_sum_to_thread0(T (&v)[NV]) {
  __shared__ T s_w[NV][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = warp_allsum(v[m]);
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < NV; ++m) s_w[m][w] = v[m];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      T t = lane < nw ? s_w[m][lane] : T(0);
      v[m] = warp_allsum(t);
    }
  }
}

// Static shared staging buffer for kernels whose groups may hold up to
// kMaxGroupBlocks blocks (a single definition, so all uses in a kernel
// share it). Kernels with dynamic shared memory carve their own instead.
static __device__ __forceinline__ double* group_stage_smem() {
  __shared__ double s_stage[kMaxGroupSlots * kMaxGroupBlocks];
  return s_stage;
}

// ---------------------------------------------------------------------------
// Warp-0 group all-reduce with split block barriers. Same association as
// group_allsum (so bit-identical totals) with fewer block-wide waits: the
// other warps post their warp sums and arrive (bar.arrive, no wait) on named
// barrier kBarPosted; warp 0 waits there, folds the block partial, publishes
// it with a release add on the group counter, polls the counter (every lane
// acquires), loads the nb block partials straight into registers, folds them
// and arrives on kBarTotal, where the other warps wait for the totals. Each
// block-wide phase is one arrive/wait pair instead of four full barriers.
// Named barriers 1 and 2 are reserved for it; the reuse order is safe because
// a warp arrives on one barrier only after passing the other.
// ---------------------------------------------------------------------------
constexpr int kBarPosted = 1;
constexpr int kBarTotal = 2;

__device__ __forceinline__ void named_arrive(int id, int nthreads) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

template <int NV, typename T>
__device__ __forceinline__ bool group_allsum_w0(T (&v)[NV], Group& g, int slot) {
  __shared__ T s_w[NV][32];
  __shared__ double s_tot[NV];
  __shared__ int s_ok;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nthreads = blockDim.x;
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = warp_allsum(v[m]);
  if (w != 0) {
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) s_w[m][w] = v[m];
    }
    named_arrive(kBarPosted, nthreads);
    named_sync(kBarTotal, nthreads);
#pragma unroll
    for (int m = 0; m < NV; ++m) v[m] = (T)s_tot[m];
    return s_ok != 0;
  }
  // Warp 0.
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < NV; ++m) s_w[m][0] = v[m];
  }
  named_sync(kBarPosted, nthreads);
  const int nw = (nthreads + 31) >> 5;
  double blk[NV];
#pragma unroll
  for (int m = 0; m < NV; ++m) blk[m] = (double)warp_allsum(lane < nw ? s_w[m][lane] : T(0));
  int ok = 1;
  if (g.nb == 1) {
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) s_tot[m] = blk[m];
    }
  } else {
    // Thread 0's count is authoritative (group_barrier advances only it).
    g.epoch = __shfl_sync(0xffffffffu, g.epoch, 0) + 1;
    const unsigned long long target = g.epoch * (unsigned long long)g.nb;
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) g.part[(size_t)(slot + m) * g.nb + g.bid] = blk[m];
      red_release_add_u64(g.counter, 1ull);
    }
    if (lane == 0) {
      uint64_t t0 = 0;
      uint32_t spins = 0;
      while (ld_acquire_u64(g.counter) < target) {
        if ((++spins & 63u) == 0) {
          if (spins == 64u) t0 = global_ns();
          if (ld_volatile_i32(g.err) != 0) { ok = 0; break; }
          if (global_ns() - t0 > g.timeout_ns) {
            atomicCAS(g.err, 0, (int)EAF_ETIMEOUT);
            ok = 0;
            break;
          }
        }
      }
    }
    // bar.warp.sync orders the other lanes' loads after lane 0's acquire.
    __syncwarp();
    ok = __shfl_sync(0xffffffffu, ok, 0);
    // Lane l folds the partials of blocks l, l + 32, ... sequentially from
    // 0.0, then the 32 lane sums are folded by the xor butterfly. Up to
    // 32 * kFew blocks, every partial of every sum is loaded in one round of
    // independent loads (one L2 round trip for all NV sums); larger groups
    // load kPer partials per lane and sum at a time.
    constexpr int kFew = 5;
    if (g.nb <= 32 * kFew) {
      double t[NV][kFew];
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        const double* p = g.part + (size_t)(slot + m) * g.nb;
#pragma unroll
        for (int u = 0; u < kFew; ++u) {
          const int b = lane + 32 * u;
          t[m][u] = b < g.nb ? __ldcg(p + b) : 0.0;
        }
      }
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        double sum = 0.0;
#pragma unroll
        for (int u = 0; u < kFew; ++u)
          if (lane + 32 * u < g.nb) sum = sum + t[m][u];
        sum = warp_allsum(sum);
        if (lane == 0) s_tot[m] = sum;
      }
    } else {
      constexpr int kPer = 8;
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        const double* p = g.part + (size_t)(slot + m) * g.nb;
        double sum = 0.0;
        for (int b0 = lane; b0 < g.nb; b0 += 32 * kPer) {
          double t[kPer];
#pragma unroll
          for (int u = 0; u < kPer; ++u) {
            const int b = b0 + 32 * u;
            t[u] = b < g.nb ? __ldcg(p + b) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kPer; ++u)
            if (b0 + 32 * u < g.nb) sum = sum + t[u];
        }
        sum = warp_allsum(sum);
        if (lane == 0) s_tot[m] = sum;
      }
    }
  }
  if (lane == 0) s_ok = ok;
  named_arrive(kBarTotal, nthreads);
  __syncwarp();
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = (T)s_tot[m];
  return ok != 0;
}

// Group all-reduce of NV sums. Per-thread and in-block sums are carried in
// T (FP32 for the mixed-precision inner solve, FP64 otherwise); block
// partials go to slots [slot, slot+NV) of the group's FP64 partial table and
// are folded in FP64. Returns false if the barrier gave up.
template <int NV, typename T, int FORM = kAllsumForm>
__device__ __forceinline__ bool group_allsum(T (&v)[NV], Group& g, int slot) {
  if (FORM == 3) return group_allsum_w0<NV, T>(v, g, slot);
  __shared__ double s_tot[NV];
  block_sum_to_thread0<NV, T>(v);
  if (g.nb == 1) {
    if (threadIdx.x == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) s_tot[m] = (double)v[m];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < NV; ++m) v[m] = (T)s_tot[m];
    __syncthreads();
    return true;
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int m = 0; m < NV; ++m) g.part[(size_t)(slot + m) * g.nb + g.bid] = (double)v[m];
  }
  const bool ok = group_barrier<(FORM >= 3 ? 1 : FORM)>(g);
  // Stage the NV x nb partials in shared memory with independent loads (all
  // in flight at once), then fold them in the fixed order: lane l of warp 0
  // sums partials l, l+32, ... sequentially, and the lanes are folded by the
  // butterfly.
  double* s_part = g.stage;
  const int total = NV * g.nb;
  const double* src = g.part + (size_t)slot * g.nb;
  for (int i0 = threadIdx.x; i0 < total; i0 += 4 * (int)blockDim.x) {
    double t[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * (int)blockDim.x;
      t[u] = i < total ? __ldcg(src + i) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * (int)blockDim.x;
      if (i < total) s_part[i] = t[u];
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      const double* p = s_part + m * g.nb;
      double s = 0.0;
      for (int b = lane; b < g.nb; b += 32) s = s + p[b];
      s = warp_allsum(s);
      if (lane == 0) s_tot[m] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = (T)s_tot[m];
  return ok;
}

// Split-phase form of group_allsum: group_arrive publishes this block's
// partials and its arrival (thread 0, after the block fold); the caller may
// then do work that neither reads the totals nor touches the reduction's
// shared buffers, and group_wait completes the reduction. Same association
// as group_allsum.
template <int NV, typename T>
__device__ __forceinline__ void group_arrive(T (&v)[NV], Group& g, int slot) {
  __shared__ double s_blk[NV];
  block_sum_to_thread0<NV, T>(v);
  if (threadIdx.x == 0) {
    if (g.nb == 1) {
#pragma unroll
      for (int m = 0; m < NV; ++m) s_blk[m] = (double)v[m];
    } else {
#pragma unroll
      for (int m = 0; m < NV; ++m) g.part[(size_t)(slot + m) * g.nb + g.bid] = (double)v[m];
      g.epoch += 1;
      red_release_add_u64(g.counter, 1ull);
    }
  }
  if (g.nb == 1) {
    __syncthreads();
#pragma unroll
    for (int m = 0; m < NV; ++m) v[m] = (T)s_blk[m];
    __syncthreads();
  }
}

template <int NV, typename T>
__device__ __forceinline__ bool group_wait(T (&v)[NV], Group& g, int slot) {
  if (g.nb == 1) return true;  // completed in group_arrive
  __shared__ int s_ok;
  __shared__ double s_tot[NV];
  if (threadIdx.x == 0) {
    const unsigned long long target = g.epoch * (unsigned long long)g.nb;
    int ok = 1;
    uint64_t t0 = 0;
    uint32_t spins = 0;
    while (ld_acquire_u64(g.counter) < target) {
      if ((++spins & 63u) == 0) {
        if (spins == 64u) t0 = global_ns();
        if (ld_volatile_i32(g.err) != 0) { ok = 0; break; }
        if (global_ns() - t0 > g.timeout_ns) {
          atomicCAS(g.err, 0, (int)EAF_ETIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  double* s_part = g.stage;
  const int total = NV * g.nb;
  const double* src = g.part + (size_t)slot * g.nb;
  for (int i0 = threadIdx.x; i0 < total; i0 += 4 * (int)blockDim.x) {
    double t[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * (int)blockDim.x;
      t[u] = i < total ? __ldcg(src + i) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * (int)blockDim.x;
      if (i < total) s_part[i] = t[u];
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      const double* p = s_part + m * g.nb;
      double s = 0.0;
      for (int b = lane; b < g.nb; b += 32) s = s + p[b];
      s = warp_allsum(s);
      if (lane == 0) s_tot[m] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = (T)s_tot[m];
  const bool ok = s_ok != 0;
  __syncthreads();
  return ok;
}

__device__ __forceinline__ double guard_small(double v) { return v > kSmall ? v : kSmall; }
__device__ __forceinline__ float guard_small(float v) {
  return v > 1.0e-30f ? v : 1.0e-30f;
}

}  // namespace eaf
