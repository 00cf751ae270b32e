// Cluster-resident FP64 CG for small systems: ONE thread-block cluster of C
// blocks (up to 16) holds the whole system in distributed shared memory for
// the whole solve, so an iteration touches global memory not at all.
//
// The solver is cg_3d_mpi (src/mod_solver_3d.f90:485-620) exactly as the
// persistent kernels of cg_f64.cu run it -- same slices (block b owns compact
// cells [b*ceil(n/C), ...)), same thread-to-cell assignment, same per-cell
// arithmetic in the reference's expression order (built with -fmad=false),
// same exit tests and NaN outcome -- with two differences in where data
// lives:
//   * each block keeps its slice of the seven coefficients (the symmetric
//     form's west, south and bottom links copied from the neighbours' east,
//     north and top links once, at load), of x, r, z, q and of the
//     double-buffered direction in its shared memory; a neighbour cell that
//     another block owns is read from that block's shared memory
//     (ld.shared::cluster);
//   * an all-reduce is one exchange: every block writes its partial into
//     every block's shared memory and signals it, and then every thread
//     folds the C partials in rank order. The association is that of the
//     cluster all-reduce with one cluster (the oracle's plan (C, B, C)), so
//     the solve is bit-identical to cg_cluster_kernel on the same launch
//     shape and to the oracle. The signal is either a full cluster barrier
//     (the default: measured faster, 3.4 against 3.9 us per iteration at
//     12x24x16) or a remote arrival on an mbarrier of each block (release at
//     cluster scope, one arrival per block and phase, barriers
//     double-buffered by all-reduce parity).
//
// Global memory is read once (the packed system) and written once (x and
// the result). There is no global synchronisation and no wait that another
// block could leave unfinished: every block of a cluster is co-scheduled
// and reaches every cluster barrier on every path (the exit decisions depend
// only on the totals, which all blocks fold identically).
#include <math.h>

#include "cg_kernels.h"
#include "cluster_red.cuh"
#include "stencil.cuh"

namespace eaf {
namespace {

// Shared-memory arrays of a slice, in this order:
//   coefficients aP aW aE aS aN aB aT, then x r z p0 p1 q, then the six
//   neighbour addresses of every cell (32-bit shared-window addresses of the
//   neighbour's element of array 0 in its owner block, or kNoNeighbour at an
//   r or z wall), which occupy the room of three more arrays.
constexpr int kDsmArrays = 16;
enum { kAP, kAW, kAE, kAS, kAN, kAB, kAT, kX, kR, kZ, kP0, kP1, kQ, kNB };
enum { kW, kE, kS, kN, kB, kT };  // neighbour directions, stencil order
constexpr uint32_t kNoNeighbour = 0xFFFFFFFFu;

struct DsmArgs {
  MeshDims d;
  SysF64 s;      // the packed compact system (read) and x (written back)
  GroupWs ws;    // result and error word
  int max_iter;
  double tol;
  uint64_t timeout_ns;
  int chunk;     // cells per block
  FastDiv fd_chunk;
};

struct PartSmem {
  double part[2][kMaxClusterSize][kClusterSlotsNV];  // by parity, by rank
  double warp[kClusterSlotsNV][32];
  uint64_t bar[2];  // arrivals of the C blocks' partials, by parity
};

// Signalling of the exchange: mbarrier arrivals (MB) or a cluster barrier.
struct Exchange {
  int C, rank, parity;
  uint32_t phase;  // completion parity expected next, bit per barrier
  int* err;
  uint64_t timeout_ns;
};

__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(
                   cluster_addr)
               : "memory");
}
__device__ __forceinline__ bool mbar_test_cluster(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ double ld_cluster_f64(uint32_t a) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
  return v;
}

struct Dsm {
  double* base;      // this block's arrays
  uint32_t base_sa;  // its shared-window address
  int chunk, rank;
  FastDiv fd;
  __device__ __forceinline__ double* arr(int k) const { return base + (size_t)k * chunk; }
  __device__ __forceinline__ uint32_t* nb(int dir) const {
    return reinterpret_cast<uint32_t*>(base + (size_t)kNB * chunk) + (size_t)dir * chunk;
  }
  // Address (in the cluster's shared window) of array 0 at compact cell cc.
  __device__ __forceinline__ uint32_t where(int cc) const {
    const int owner = (int)fd.div((uint32_t)cc);
    const int off = cc - owner * chunk;
    return cluster_map(base_sa + 8u * (uint32_t)off, (uint32_t)owner);
  }
  // Value of array k at the neighbour whose array-0 address is a.
  __device__ __forceinline__ double at(int k, uint32_t a) const {
    return ld_cluster_f64(a + 8u * (uint32_t)k * (uint32_t)chunk);
  }
};

// Every block's partials go to every block, then each thread folds them in
// rank order (starting from rank 0's). Returns false if a bounded wait gave
// up (then every thread of the block returns false).
template <int NV, bool MB>
__device__ __forceinline__ bool dsm_allsum(double (&v)[NV], PartSmem& ps, Exchange& x) {
  const int C = x.C, rank = x.rank, parity = x.parity;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nthreads = blockDim.x;
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = warp_allsum(v[m]);
  if (w != 0) {
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) ps.warp[m][w] = v[m];
    }
    named_arrive(kBarPosted, nthreads);
  } else {
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) ps.warp[m][0] = v[m];
    }
    named_sync(kBarPosted, nthreads);
    const int nw = (nthreads + 31) >> 5;
    double blk[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) blk[m] = warp_allsum(lane < nw ? ps.warp[m][lane] : 0.0);
    if (lane < C) {
      const uint32_t dst = cluster_map(smem_addr(&ps.part[parity][rank][0]), (uint32_t)lane);
#pragma unroll
      for (int m = 0; m < NV; ++m) st_cluster_f64(dst + 8u * m, blk[m]);
      if (MB) mbar_arrive_remote(cluster_map(smem_addr(&ps.bar[parity]), (uint32_t)lane));
    }
    __syncwarp();
  }
  bool ok = true;
  if (MB) {
    // Every thread acquires the C arrivals itself (bounded wait).
    const uint32_t a = smem_addr(&ps.bar[parity]);
    const uint32_t want = (x.phase >> parity) & 1u;
    if (!mbar_test_cluster(a, want)) {
      const uint64_t t0 = global_ns();
      uint32_t spins = 0;
      while (!mbar_test_cluster(a, want)) {
        if ((++spins & 255u) == 0) {
          if (ld_volatile_i32(x.err) != 0) { ok = false; break; }
          if (global_ns() - t0 > x.timeout_ns) {
            atomicCAS(x.err, 0, (int)EAF_ETIMEOUT);
            ok = false;
            break;
          }
        }
      }
    }
    x.phase ^= 1u << parity;
    ok = __syncthreads_and(ok) != 0;
  } else {
    cluster_sync_all();
  }
  x.parity ^= 1;
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    double t = ps.part[parity][0][m];
    for (int r = 1; r < C; ++r) t = t + ps.part[parity][r][m];
    v[m] = t;
  }
  return ok;
}

// y = A x at own cell o, the reference's expression order; the coefficients
// are this block's copies, neighbour values come from xv(neighbour address)
// (a missing neighbour -- r or z wall -- is skipped in the symmetric form and
// multiplies a zero value in the general form, as in apply_row_with).
template <bool SYM, typename XF>
__device__ __forceinline__ double dsm_row(const Dsm& m, int o, double xc, XF xv) {
  const uint32_t w = m.nb(kW)[o], e = m.nb(kE)[o], so = m.nb(kS)[o];
  const uint32_t no = m.nb(kN)[o], bo = m.nb(kB)[o], t = m.nb(kT)[o];
  double y = m.arr(kAP)[o] * xc;
  if (SYM) {
    if (w != kNoNeighbour) y = y - m.arr(kAW)[o] * xv(w);
    if (e != kNoNeighbour) y = y - m.arr(kAE)[o] * xv(e);
    y = y - m.arr(kAS)[o] * xv(so);
    y = y - m.arr(kAN)[o] * xv(no);
    if (bo != kNoNeighbour) y = y - m.arr(kAB)[o] * xv(bo);
    if (t != kNoNeighbour) y = y - m.arr(kAT)[o] * xv(t);
  } else {
    const double xw = w != kNoNeighbour ? xv(w) : 0.0;
    const double xe = e != kNoNeighbour ? xv(e) : 0.0;
    const double xb = bo != kNoNeighbour ? xv(bo) : 0.0;
    const double xt = t != kNoNeighbour ? xv(t) : 0.0;
    y = y - m.arr(kAW)[o] * xw;
    y = y - m.arr(kAE)[o] * xe;
    y = y - m.arr(kAS)[o] * xv(so);
    y = y - m.arr(kAN)[o] * xv(no);
    y = y - m.arr(kAB)[o] * xb;
    y = y - m.arr(kAT)[o] * xt;
  }
  return y;
}

template <bool SYM, bool MB>
__device__ void dsm_body(const DsmArgs& a, const Dsm& m, PartSmem& ps, int C) {
  const MeshDims& d = a.d;
  const SysF64& s = a.s;
  const int rank = m.rank;
  Exchange xc;
  xc.C = C;
  xc.rank = rank;
  xc.parity = 0;
  xc.phase = 0;
  xc.err = a.ws.err;
  xc.timeout_ns = a.timeout_ns;
  const int begin = min(d.n, rank * a.chunk);
  const int end = min(d.n, begin + a.chunk);
  const int B = blockDim.x;

  // Load the slice; the symmetric form's west/south/bottom links are the
  // neighbours' east/north/top links (zero at the r and z walls, where the
  // solver skips them).
  for (int c = begin + (int)threadIdx.x; c < end; c += B) {
    const int o = c - begin;
    int i, j, k;
    cell_ijk(d, c, i, j, k);
    const int cs = j > 0 ? c - d.nr : c + (d.nth - 1) * d.nr;
    m.arr(kAP)[o] = s.aP[c];
    m.arr(kAE)[o] = s.aE[c];
    m.arr(kAN)[o] = s.aN[c];
    m.arr(kAT)[o] = s.aT[c];
    if (SYM) {
      m.arr(kAW)[o] = i > 0 ? s.aE[c - 1] : 0.0;
      m.arr(kAS)[o] = s.aN[cs];
      m.arr(kAB)[o] = k > 0 ? s.aT[c - d.plane] : 0.0;
    } else {
      m.arr(kAW)[o] = s.aW[c];
      m.arr(kAS)[o] = s.aS[c];
      m.arr(kAB)[o] = s.aB[c];
    }
    m.arr(kX)[o] = s.x[c];
    const int cn = j < d.nth - 1 ? c + d.nr : c - (d.nth - 1) * d.nr;
    m.nb(kW)[o] = i > 0 ? m.where(c - 1) : kNoNeighbour;
    m.nb(kE)[o] = i < d.nr - 1 ? m.where(c + 1) : kNoNeighbour;
    m.nb(kS)[o] = m.where(cs);
    m.nb(kN)[o] = m.where(cn);
    m.nb(kB)[o] = k > 0 ? m.where(c - d.plane) : kNoNeighbour;
    m.nb(kT)[o] = k < d.nz - 1 ? m.where(c + d.plane) : kNoNeighbour;
  }
  // Preamble (src/mod_solver_3d.f90:515-530): ||Su||, z = r/max(|aP|,SMALL),
  // p = z, r.z and r.r.
  double v3[3] = {0.0, 0.0, 0.0};
  for (int c = begin + (int)threadIdx.x; c < end; c += B) {
    const int o = c - begin;
    const double bv = s.b[c], rv = s.r[c];
    const double zv = rv / guard_small(fabs(s.aP[c]));
    m.arr(kR)[o] = rv;
    m.arr(kZ)[o] = zv;
    m.arr(kP0)[o] = zv;
    v3[0] = v3[0] + bv * bv;
    v3[1] = v3[1] + rv * rv;
    v3[2] = v3[2] + rv * zv;
  }
  bool ok = dsm_allsum<3, MB>(v3, ps, xc);
  const double bnorm = sqrt(v3[0]);
  double residual = 0.0;
  int n_iter = 0;
  bool nan_fill = false;
  if (ok && !(bnorm < kSmall)) {
    double rz = v3[2];
    double beta = 0.0;
    residual = sqrt(v3[1]) / bnorm;
    if (residual != residual && a.max_iter >= 1) nan_fill = true;
    for (int iter = 1; iter <= a.max_iter && !nan_fill; ++iter) {
      // Phase A: p = z + beta p_old fused with q = A p and p.q.
      const int kcur = (iter & 1) ? kP0 : kP1;
      const int kold = (iter & 1) ? kP1 : kP0;
      double* pcur = m.arr(kcur);
      double* q = m.arr(kQ);
      double v1[1] = {0.0};
      if (iter == 1) {
        auto xv = [&m, kcur](uint32_t na) { return m.at(kcur, na); };
        for (int c = begin + (int)threadIdx.x; c < end; c += B) {
          const int o = c - begin;
          const double pc = pcur[o];
          const double qv = dsm_row<SYM>(m, o, pc, xv);
          q[o] = qv;
          v1[0] = v1[0] + pc * qv;
        }
      } else {
        const double bt = beta;
        auto pnew = [&m, kold, bt](uint32_t na) { return m.at(kZ, na) + bt * m.at(kold, na); };
        const double* z = m.arr(kZ);
        const double* pold = m.arr(kold);
        for (int c = begin + (int)threadIdx.x; c < end; c += B) {
          const int o = c - begin;
          const double pc = z[o] + bt * pold[o];
          const double qv = dsm_row<SYM>(m, o, pc, pnew);
          pcur[o] = pc;
          q[o] = qv;
          v1[0] = v1[0] + pc * qv;
        }
      }
      if (!(ok = dsm_allsum<1, MB>(v1, ps, xc))) break;
      const double pq = v1[0];
      if (fabs(pq) < kSmall) break;
      const double alpha = rz / pq;
      // Phase B: phi += alpha p; r -= alpha q; r.r; z and r.z (:538-553)
      double v2[2] = {0.0, 0.0};
      {
        double* x = m.arr(kX);
        double* r = m.arr(kR);
        double* z = m.arr(kZ);
        const double* aP = m.arr(kAP);
        for (int c = begin + (int)threadIdx.x; c < end; c += B) {
          const int o = c - begin;
          const double xn = x[o] + alpha * pcur[o];
          const double rn = r[o] - alpha * q[o];
          const double zv = rn / guard_small(fabs(aP[o]));
          x[o] = xn;
          r[o] = rn;
          z[o] = zv;
          v2[0] = v2[0] + rn * rn;
          v2[1] = v2[1] + rn * zv;
        }
      }
      if (!(ok = dsm_allsum<2, MB>(v2, ps, xc))) break;
      residual = sqrt(v2[0]) / bnorm;
      n_iter = iter;
      if (residual < a.tol) break;
      if (residual != residual && iter < a.max_iter) { nan_fill = true; break; }
      beta = v2[1] / guard_small(rz);
      rz = v2[1];
    }
  }
  // x back to global memory for the unpack kernel.
  const double qnan = __longlong_as_double(0x7ff8000000000000ll);
  for (int c = begin + (int)threadIdx.x; c < end; c += B)
    s.x[c] = nan_fill ? qnan : m.arr(kX)[c - begin];
  if (nan_fill) {
    residual = qnan;
    n_iter = a.max_iter;
  }
  if (rank == 0 && threadIdx.x == 0) {
    SolveResult* res = a.ws.result;
    const int err = ld_volatile_i32(a.ws.err);
    res->status = err != 0 ? err : (isfinite(residual) ? EAF_OK : EAF_ENONFINITE);
    res->n_iter = n_iter;
    res->n_outer = 0;
    res->sym = SYM ? 1 : 0;
    res->residual = residual;
    res->bnorm = bnorm;
  }
}

template <bool MB>
__global__ void __launch_bounds__(1024, 1) cg_dsm_kernel(DsmArgs a) {
  extern __shared__ __align__(16) double dsm_smem[];
  __shared__ __align__(8) PartSmem ps;
  Dsm m;
  m.base = dsm_smem;
  m.base_sa = smem_addr(dsm_smem);
  m.chunk = a.chunk;
  m.rank = (int)cluster_ctarank();
  m.fd = a.fd_chunk;
  const int C = (int)cluster_nctarank();
  if (MB && threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&ps.bar[0])), "r"(C)
                 : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&ps.bar[1])), "r"(C)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // Every block has started (and initialised its barriers) before any
  // block addresses another's memory.
  cluster_sync_all();
  if (*a.s.asym == 0)
    dsm_body<true, MB>(a, m, ps, C);
  else
    dsm_body<false, MB>(a, m, ps, C);
  // No block leaves while another may still address its shared memory.
  cluster_sync_all();
}

size_t dsm_smem_bytes(int chunk) { return (size_t)kDsmArrays * chunk * sizeof(double); }

}  // namespace

int dsm_max_cells(int cluster) {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
      cudaSuccess)
    return 0;
  const long long avail = (long long)optin - (long long)sizeof(PartSmem) - 1024;
  if (avail <= 0) return 0;
  const long long per_block = avail / (kDsmArrays * (long long)sizeof(double));
  return (int)(per_block * cluster);
}

bool dsm_can_launch(long long n, int block, int cluster) {
  if (cluster < 1 || cluster > kMaxClusterSize || block < 32 || block > 1024 ||
      block % 32 != 0 || n > dsm_max_cells(cluster))
    return false;
  const int chunk = (int)((n + cluster - 1) / cluster);
  const size_t smem = dsm_smem_bytes(chunk);
  const void* k = (const void*)cg_dsm_kernel<false>;
  std::lock_guard<std::mutex> attr_lock(launch_attr_mutex());
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess ||
      (cluster > 8 &&
       cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
           cudaSuccess)) {
    (void)cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int count = 0;
  if (cudaOccupancyMaxActiveClusters(&count, k, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return count >= 1;
}

cudaError_t launch_cg_f64_dsm(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                              int max_iter, double tol, int block, int cluster,
                              cudaStream_t st, int signal, uint64_t timeout_ns) {
  if (cluster < 1 || cluster > kMaxClusterSize || block < 32 || block > 1024 ||
      block % 32 != 0 || d.n > dsm_max_cells(cluster))
    return cudaErrorInvalidValue;
  DsmArgs a;
  a.d = d;
  a.s = s;
  a.ws = ws;
  a.max_iter = max_iter;
  a.tol = tol;
  a.timeout_ns = timeout_ns;
  a.chunk = (d.n + cluster - 1) / cluster;
  a.fd_chunk = FastDiv((uint32_t)a.chunk);
  const size_t smem = dsm_smem_bytes(a.chunk);
  const void* k = signal == kDsmSignalMbarrier ? (const void*)cg_dsm_kernel<true>
                                                : (const void*)cg_dsm_kernel<false>;
  std::lock_guard<std::mutex> attr_lock(launch_attr_mutex());
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e == cudaSuccess && cluster > 8)
    e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  (void)cudaGetLastError();  // report this launch's error, not an older one
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {&a};
  return cudaLaunchKernelExC(&cfg, k, args);
}

}  // namespace eaf
