// Slot-signalled all-reduces (the value in a slot is its own signal: slots
// hold a signalling-NaN marker until written):
//   * cluster_allsum: the grid of a persistent solver launched as clusters of
//     C co-scheduled blocks (thread-block clusters, up to 16 per cluster),
//     with the group reduction split into a distributed-shared-memory stage
//     inside each cluster and a global stage among the cluster leaders only;
//   * group_allsum_slots (further below): the flat grid's p.q all-reduce
//     without a release.
//
//   1. every block folds its partial as the group all-reduce does (warp
//      butterflies, warp 0 folds the warp sums) and warp 0 writes it into the
//      leader block's (cluster rank 0) shared memory (st.shared::cluster);
//   2. cluster barrier (release/acquire at cluster scope);
//   3. the leader's warp 0 folds the C block partials in rank order; with
//      more than one cluster it publishes the cluster partial in global
//      memory and reads every leader's partial straight from its slot (the
//      value is the signal: slots hold a signalling-NaN marker until written,
//      which no arithmetic produces), then folds them in a fixed order;
//   4. the leader writes the totals (and an ok flag) into every block's
//      shared memory; cluster barrier; every thread reads them.
//
// Association (restated by the oracle's cluster plan): block partials as in
// group_allsum; cluster partial cp = (((p_0 + p_1) + p_2) + ...) over the
// cluster's blocks in rank order; one cluster: total = cp; otherwise lane l
// of the leader warp sums cp_l, cp_{l+32}, ... sequentially from 0.0 and the
// 32 lane sums are folded by the xor butterfly. With C = 1 this is exactly
// the association of group_allsum: a flat grid whose all-reduce polls the
// partials themselves instead of an arrival counter (EAF_CG_KERNEL_SLOTS).
//
// Memory ordering. Block writes are ordered before the block's cluster
// barrier arrival (release, cluster scope); the leader acquires them at the
// barrier, issues fence.acq_rel.gpu and stores its partials (release
// pattern); a reader's relaxed polls that observe every value are followed
// by fence.acq_rel.gpu (acquire pattern); the second cluster barrier carries
// that to the reader's cluster. So everything any block wrote before an
// all-reduce happens before what every block does after it, as for the
// group barrier.
//
// Slots rotate over three sets: at all-reduce e a leader writes set e % 3 and
// first resets its own slot of set (e + 1) % 3, last written at e - 2 and
// read by every leader before it published e - 1. The launcher fills all
// slots with the marker before the launch.
//
// Waits: the leaders' polls are bounded by the group timeout and stop when
// the shared error word is set; the cluster barriers cannot wait forever
// because every block of a cluster (co-scheduled by construction) reaches
// each of them on every path: the exit decisions of a solve depend only on
// the totals and the ok flag, which are the same in all blocks of a
// cluster.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cg_common.cuh"

namespace eaf {

constexpr int kMaxClusterSize = 16;
constexpr int kPerLane = 5;            // leaders' slots a lane reads
constexpr int kMaxClusters = 32 * kPerLane;
constexpr int kClusterSlotsNV = 4;     // sums per all-reduce, at most
constexpr int kClusterSets = 3;
// Signalling NaN (quiet bit clear, payload nonzero): the empty-slot marker.
constexpr unsigned long long kSlotMarker = 0x7FF4DEADBEEF0001ull;

// Doubles of the global slot table for `ncl` clusters.
__host__ __device__ constexpr size_t cluster_slot_doubles(int ncl) {
  return (size_t)kClusterSets * kClusterSlotsNV * (size_t)ncl;
}

struct ClusterGroup {
  double* slots;      // [set][m][cluster], global, marker-filled before launch
  int* err;           // shared error word
  uint64_t timeout_ns;
  int nb, bid;        // blocks of the grid, this block's index
  int C, rank;        // cluster size, rank of this block in its cluster
  int ncl, cl;        // clusters, this block's cluster
  unsigned epoch;     // all-reduces completed (uniform)
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t cluster_map(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster_f64(uint32_t a, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
// Full cluster barrier; every thread of every block of the cluster takes
// part. Callers keep each warp converged at it.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_nctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t nclusters_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool is_marker(double v) {
  return (unsigned long long)__double_as_longlong(v) == kSlotMarker;
}

__device__ __forceinline__ ClusterGroup make_cluster_group(double* slots, int* err,
                                                           uint64_t timeout_ns) {
  ClusterGroup g;
  g.slots = slots;
  g.err = err;
  g.timeout_ns = timeout_ns;
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.C = (int)cluster_nctarank();
  g.rank = (int)cluster_ctarank();
  g.ncl = (int)nclusters_x();
  g.cl = (int)cluster_id_x();
  g.epoch = 0;
  return g;
}

// Shared-memory state of one block (static, one instance per kernel).
struct ClusterSmem {
  double gather[kMaxClusterSize][kClusterSlotsNV];  // leader: block partials by rank
  double tot[kClusterSlotsNV];                      // totals written by the leader
  double warp[kClusterSlotsNV][32];                 // warp sums of this block
  int ok;
};
static __device__ __forceinline__ ClusterSmem& cluster_smem() {
  __shared__ ClusterSmem s;
  return s;
}

// ---------------------------------------------------------------------------
// One-sum group all-reduce without a release, for the flat solver's p.q.
// Nothing a block writes in the stencil phase is read by another block before
// the r.r / r.z all-reduce that follows the update phase, and that one keeps
// its release and acquire; so this all-reduce only has to carry the partials,
// and its cost is no longer a release that waits for the SM's outstanding
// stores. Each block's warp 0 folds its partial as group_allsum_w0 does, then
// lane 0 writes it with a relaxed store into its slot of the set of this
// iteration and adds 1 to the group counter with a relaxed add (a doorbell,
// no ordering). Lane 0 polls the counter (relaxed) up to the all-reduce's
// target; then every lane loads its slots (blocks l, l+32, ...) with relaxed
// loads, re-loading any that still holds the marker (the value is the
// signal: a signalling NaN no arithmetic produces), and the partials are
// folded in group_allsum_w0's order, so the totals are bit-identical to it.
//
// Slots: two sets of nb doubles at `slots`, used alternately by the group's
// successive p.q all-reduces (g.pq_seq counts them, so the alternation also
// holds across several solves by one group), filled with the marker before
// the launch. At its s-th p.q all-reduce a block first resets its slot of
// the other set, last written at s - 1: every block read that set before it
// arrived at the next all-reduce with a release (the r.r / r.z of the same
// iteration, or the preamble of a following solve), whose release/acquire
// orders those reads before this reset; the release/acquire all-reduce
// between s and s + 1 orders the reset before the reads of s + 1.
// Counter epochs are shared with group_allsum_w0: every block adds 1 per
// all-reduce, so the count reaches epoch * nb only when all have.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void red_relaxed_add_u64(unsigned long long* p,
                                                    unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ bool group_allsum_slots(double (&v)[1], Group& g, double* slots) {
  const int seq = ++g.pq_seq;
  __shared__ double s_w[32];
  __shared__ double s_tot;
  __shared__ int s_ok;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nthreads = blockDim.x;
  v[0] = warp_allsum(v[0]);
  if (w != 0) {
    if (lane == 0) s_w[w] = v[0];
    named_arrive(kBarPosted, nthreads);
    named_sync(kBarTotal, nthreads);
    v[0] = s_tot;
    return s_ok != 0;
  }
  if (lane == 0) s_w[0] = v[0];
  named_sync(kBarPosted, nthreads);
  const int nw = (nthreads + 31) >> 5;
  const double blk = warp_allsum(lane < nw ? s_w[lane] : 0.0);
  int ok = 1;
  if (g.nb == 1) {
    if (lane == 0) s_tot = blk;
  } else {
    g.epoch = __shfl_sync(0xffffffffu, g.epoch, 0) + 1;
    const unsigned long long target = g.epoch * (unsigned long long)g.nb;
    double* cur = slots + (size_t)(seq & 1) * g.nb;
    double* other = slots + (size_t)((seq + 1) & 1) * g.nb;
    if (lane == 0) {
      st_relaxed_f64(other + g.bid, __longlong_as_double((long long)kSlotMarker));
      st_relaxed_f64(cur + g.bid, blk);
      red_relaxed_add_u64(g.counter, 1ull);
      uint64_t t0 = 0;
      uint32_t spins = 0;
      while (ld_relaxed_u64(g.counter) < target) {
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
    ok = __shfl_sync(0xffffffffu, ok, 0);
    double sum = 0.0;
    if (ok) {
      double t[kPerLane];
#pragma unroll
      for (int u = 0; u < kPerLane; ++u) {
        const int b = lane + 32 * u;
        t[u] = b < g.nb ? ld_relaxed_f64(cur + b) : 0.0;
      }
      // A partial whose doorbell overtook it: load it again (bounded).
      uint64_t t0 = 0;
      uint32_t spins = 0;
      bool mine = true;
#pragma unroll
      for (int u = 0; u < kPerLane; ++u) mine = mine && !is_marker(t[u]);
      while (!__all_sync(0xffffffffu, mine)) {
#pragma unroll
        for (int u = 0; u < kPerLane; ++u) {
          const int b = lane + 32 * u;
          if (is_marker(t[u])) t[u] = ld_relaxed_f64(cur + b);
        }
        mine = true;
#pragma unroll
        for (int u = 0; u < kPerLane; ++u) mine = mine && !is_marker(t[u]);
        if ((++spins & 15u) == 0) {
          if (spins == 16u) t0 = global_ns();
          int bad = 0;
          if (lane == 0) {
            if (ld_volatile_i32(g.err) != 0) {
              bad = 1;
            } else if (global_ns() - t0 > g.timeout_ns) {
              atomicCAS(g.err, 0, (int)EAF_ETIMEOUT);
              bad = 1;
            }
          }
          if (__shfl_sync(0xffffffffu, bad, 0)) {
            ok = 0;
            break;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < kPerLane; ++u)
        if (lane + 32 * u < g.nb) sum = sum + t[u];
    }
    sum = warp_allsum(sum);
    if (lane == 0) s_tot = sum;
  }
  if (lane == 0) s_ok = ok;
  named_arrive(kBarTotal, nthreads);
  __syncwarp();
  v[0] = s_tot;
  return ok != 0;
}

template <int NV, typename T>
__device__ __forceinline__ bool cluster_allsum(T (&v)[NV], ClusterGroup& g) {
  static_assert(NV <= kClusterSlotsNV, "too many sums for one cluster all-reduce");
  ClusterSmem& sm = cluster_smem();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nthreads = blockDim.x;
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = warp_allsum(v[m]);
  if (w != 0) {
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) sm.warp[m][w] = (double)v[m];
    }
    named_arrive(kBarPosted, nthreads);
  } else {
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) sm.warp[m][0] = (double)v[m];
    }
    named_sync(kBarPosted, nthreads);
    const int nw = (nthreads + 31) >> 5;
    double blk[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) blk[m] = warp_allsum(lane < nw ? sm.warp[m][lane] : 0.0);
    if (lane == 0) {
      const uint32_t dst = cluster_map(smem_addr(&sm.gather[g.rank][0]), 0);
#pragma unroll
      for (int m = 0; m < NV; ++m) st_cluster_f64(dst + 8u * m, blk[m]);
    }
    __syncwarp();
  }
  cluster_sync_all();
  g.epoch += 1;
  if (g.rank == 0 && w == 0) {
    double cp[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      cp[m] = sm.gather[0][m];
      for (int r = 1; r < g.C; ++r) cp[m] = cp[m] + sm.gather[r][m];
    }
    int ok = 1;
    double tot[NV];
    if (g.ncl == 1) {
#pragma unroll
      for (int m = 0; m < NV; ++m) tot[m] = cp[m];
    } else {
      const int set = (int)(g.epoch % kClusterSets);
      const int old = (int)((g.epoch + 1) % kClusterSets);
      const size_t stride = (size_t)g.ncl;
      double* cur = g.slots + (size_t)set * kClusterSlotsNV * stride;
      if (lane == 0) {
        double* prev = g.slots + (size_t)old * kClusterSlotsNV * stride;
        const double marker = __longlong_as_double((long long)kSlotMarker);
#pragma unroll
        for (int m = 0; m < NV; ++m) st_relaxed_f64(prev + m * stride + g.cl, marker);
        fence_acq_rel_gpu();
#pragma unroll
        for (int m = 0; m < NV; ++m) st_relaxed_f64(cur + m * stride + g.cl, cp[m]);
      }
      // lane l reads the partials of clusters l, l + 32, ...
      double got[kPerLane][NV];
      uint64_t t0 = 0;
      uint32_t spins = 0;
      bool done = false;
      while (true) {
        bool mine = true;
#pragma unroll
        for (int u = 0; u < kPerLane; ++u) {
          const int c = lane + 32 * u;
#pragma unroll
          for (int m = 0; m < NV; ++m) {
            got[u][m] = c < g.ncl ? ld_relaxed_f64(cur + m * stride + c) : 0.0;
            mine = mine && !is_marker(got[u][m]);
          }
        }
        done = __all_sync(0xffffffffu, mine);
        if (done) break;
        if ((++spins & 15u) == 0) {
          if (spins == 16u) t0 = global_ns();
          int bad = 0;
          if (lane == 0) {
            if (ld_volatile_i32(g.err) != 0) {
              bad = 1;
            } else if (global_ns() - t0 > g.timeout_ns) {
              atomicCAS(g.err, 0, (int)EAF_ETIMEOUT);
              bad = 1;
            }
          }
          if (__shfl_sync(0xffffffffu, bad, 0)) break;
        }
      }
      fence_acq_rel_gpu();
      ok = done ? 1 : 0;
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        double s = 0.0;
#pragma unroll
        for (int u = 0; u < kPerLane; ++u)
          if (lane + 32 * u < g.ncl) s = s + got[u][m];
        tot[m] = warp_allsum(s);
      }
    }
    if (lane < g.C) {
      const uint32_t dst = cluster_map(smem_addr(&sm.tot[0]), (uint32_t)lane);
#pragma unroll
      for (int m = 0; m < NV; ++m) st_cluster_f64(dst + 8u * m, tot[m]);
      const uint32_t dok = cluster_map(smem_addr(&sm.ok), (uint32_t)lane);
      asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(dok), "r"(ok) : "memory");
    }
    __syncwarp();
  }
  cluster_sync_all();
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = (T)sm.tot[m];
  return sm.ok != 0;
}

}  // namespace eaf
