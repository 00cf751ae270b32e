// Plain FP64 Jacobi-preconditioned CG for the SIMPLE pressure correction:
// a B200 restatement of cg_3d_mpi (src/mod_solver_3d.f90:485-620).
//
// Built with -fmad=false: every a*b+c below is rounded twice, as the
// reference's default gfortran build computes it, so the stencil, the
// updates and the preconditioner match the reference cell by cell and only
// the association of the scalar dot products differs.
//
// One persistent cooperative launch runs the whole solve. Each block owns a
// contiguous slice of cells (compact layout, cg_common.cuh) in every phase;
// an iteration is two phases, each closed by a group all-reduce:
//   A  p_new = z + beta p_old (own cells into the other p buffer; the six
//      neighbours' p_new recomputed from their stored z and p_old),
//      q = A p_new, partial p.q                    -> all-reduce p.q
//   B  x += alpha p, r -= alpha q, z = r / max(|aP|, SMALL) stored,
//      partial r.r and r.z                         -> all-reduce (r.r, r.z)
// The scalar recurrences (alpha, beta, residual, exit tests) are evaluated
// redundantly and bit-identically by every block.
//
// Forms: cg_f64_kernel (per-thread loads), cg_keep_kernel (the same with
// each block's own cells' x, r, aP and q kept in shared memory for the whole
// solve), cg_stream_kernel (operands staged by bulk copies), cg_cluster_kernel
// (grid of thread-block clusters), cg1_f64_kernel (one all-reduce per
// iteration, rearranged recurrences) and batch_f64_kernel (many systems on
// lanes of one launch). On flat grids of up to 160 blocks the p.q all-reduce
// carries no release (group_allsum_slots in cluster_red.cuh).
#include <math.h>

#include "cg_kernels.h"
#include "cluster_red.cuh"
#include "stencil.cuh"
#include "stream_stage.cuh"

namespace eaf {

MeshDims make_dims(int nr, int nth, int nz) {
  MeshDims d;
  d.nr = nr;
  d.nth = nth;
  d.nz = nz;
  d.plane = nr * nth;
  d.n = nr * nth * nz;
  d.fd_nr = FastDiv((uint32_t)nr);
  d.fd_nth = FastDiv((uint32_t)nth);
  return d;
}

namespace {

// Bulk L2 prefetch (the TMA unit's cp.async.bulk.prefetch.L2) of cells
// [lo, hi) of array a, clamped to [0, n) and to 16-byte boundaries inside the
// array; a hint with no register or ordering cost.
__device__ __forceinline__ void l2_prefetch_cells(const double* a, int lo, int hi, int n) {
  lo = max(lo, 0);
  hi = min(hi, n);
  if (hi <= lo) return;
  const uintptr_t base = (uintptr_t)a;
  const uintptr_t b = ((uintptr_t)(a + lo)) & ~(uintptr_t)15;
  uintptr_t e = ((uintptr_t)(a + hi) + 15) & ~(uintptr_t)15;
  const uintptr_t end = (base + (uintptr_t)n * 8) & ~(uintptr_t)15;
  if (e > end) e = end;
  if (b < base || e <= b) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"((unsigned)(e - b))
               : "memory");
}

// The group all-reduce of a persistent solver, by the kind of group: a flat
// group of co-resident blocks (one global stage over all blocks) or a grid
// of thread-block clusters (shared-memory stage per cluster, global stage
// among cluster leaders).
template <int NV>
__device__ __forceinline__ bool allsum(double (&v)[NV], Group& g, int slot) {
  return group_allsum<NV>(v, g, slot);
}
template <int NV>
__device__ __forceinline__ bool allsum(double (&v)[NV], ClusterGroup& g, int) {
  return cluster_allsum<NV>(v, g);
}

// Doubles a cell the KEEP form holds in shared memory: x, r, aP, q.
constexpr int kKeepArrays = 4;
// Partial-table slots of the flat solver: 0-2 the preamble's sums, 3 p.q in
// the counter form, 4-5 r.r and r.z, 6-7 the two p.q slot sets of
// group_allsum_slots (the table holds 8 doubles per block).
constexpr int kPqSlotOffset = 6;

struct CgArgs {
  MeshDims d;
  SysF64 s;
  GroupWs ws;
  int max_iter;
  double tol;
  uint64_t timeout_ns;
};

// Loops over this thread's cells of the block slice in rounds of U cells
// (cell c0 + u*B of round c0). Every round first loads what all U cells need
// (indices clamped into the slice, so no branch guards a load and all loads
// of the round are in flight together), then computes and stores with the
// out-of-slice lanes masked. Dead lanes add +0.0 to the dot sums, which
// leaves them bit-identical to sums over the live cells alone.

// U: cells per thread per round of the streaming phases; UA: of the stencil
// phase. Kernels pick them by their register budget. PF: threads 0..7 of the
// block prefetch the block's next round of every streamed array into L2
// (one bulk prefetch per array), for meshes whose working set exceeds L2.
// KEEP: the thread's own cells' x, r, aP and this iteration's q = A p stay
// in the block's shared memory (`keep`, kKeepArrays x slice-length doubles)
// for the whole solve: the stencil takes the cell's own aP from there, the
// update phase reads only the new direction from global memory (the
// stencil phase stored it there for the neighbours), q is never stored
// globally, and x goes back to global memory once, at the end. A thread
// visits the same cells in both phases (and every iteration), so no other
// thread ever reads what it keeps; the arithmetic and the order of every
// sum are unchanged. The direction itself is not kept: the L1 room it
// would take costs the stencil phase more than the update phase gains.
// PQS: the p.q all-reduce of a flat grid (Group) runs without a release,
// through the slot sets at part + kPqSlotOffset * nb (group_allsum_slots),
// up to 32 * kPerLane blocks; larger grids use the counter form.
template <bool SYM, int U, int UA, bool PF, class G, bool KEEP = false, bool PQS = false>
__device__ void cg_body(const CgArgs& a, G& g, double* keep = nullptr) {
  const MeshDims& d = a.d;
  const SysF64& s = a.s;
  const Slice own = own_slice(d.n, g.nb, g.bid);
  const int slen = own.end - own.begin;
  double* __restrict__ kx = keep;
  double* __restrict__ kr = keep + (size_t)1 * (KEEP ? slen : 0);
  double* __restrict__ kd = keep + (size_t)2 * (KEEP ? slen : 0);
  double* __restrict__ kq = keep + (size_t)3 * (KEEP ? slen : 0);
  const Coefs<double> A = coefs_of<double>(s.aP, s.aE, s.aN, s.aT, s.aW, s.aS, s.aB);
  const double* __restrict__ aP = s.aP;
  const double* __restrict__ b = s.b;
  double* __restrict__ x = s.x;
  double* __restrict__ r = s.r;
  double* __restrict__ z = s.z;
  double* __restrict__ q = s.q;
  const int B = blockDim.x;
  const int last = own.end - 1;

  // Preamble (src/mod_solver_3d.f90:515-530): ||Su||, z = r/max(|aP|,SMALL),
  // pv = z, r.z and r.r in one pass.
  double v3[3] = {0.0, 0.0, 0.0};
  {
    double* __restrict__ p0 = s.p;
    for (int c0 = own.begin + (int)threadIdx.x; c0 < own.end; c0 += B * U) {
      double bv[U], rv[U], dv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int c = min(c0 + u * B, last);
        bv[u] = b[c];
        rv[u] = r[c];
        dv[u] = aP[c];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool live = c0 + u * B < own.end;
        const double zv = rv[u] / guard_small(fabs(dv[u]));
        if (live) p0[c0 + u * B] = zv;
        if (KEEP && live) {
          const int o = c0 + u * B - own.begin;
          kx[o] = x[c0 + u * B];
          kr[o] = rv[u];
          kd[o] = dv[u];
        }
        v3[0] = v3[0] + (live ? bv[u] * bv[u] : 0.0);
        v3[1] = v3[1] + (live ? rv[u] * rv[u] : 0.0);
        v3[2] = v3[2] + (live ? rv[u] * zv : 0.0);
      }
    }
  }
  bool ok = allsum<3>(v3, g, 0);
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
      // Phase A: pv = z + beta pv (src/mod_solver_3d.f90:556-558) fused with
      // q = A pv and p.q (:533-534). The new direction goes to the other
      // buffer; neighbours' new values are formed here from their stored z
      // and old direction (both final since the last barrier), so no
      // barrier separates the update from the stencil. Iteration 1 uses
      // pv = z from the preamble as is.
      const double* __restrict__ pold = (iter & 1) ? s.p2 : s.p;
      double* __restrict__ pcur = (iter & 1) ? s.p : s.p2;
      double v1[1] = {0.0};
      if (iter == 1) {
        for (int c0 = own.begin + (int)threadIdx.x; c0 < own.end; c0 += B * UA) {
          if (PF && threadIdx.x < 6) {
            const int nl = c0 - (int)threadIdx.x + B * UA, nh = min(nl + B * UA, own.end);
            const double* arr[6] = {pcur, aP, A.aE, A.aN, A.aT, pcur};
            const int off = threadIdx.x == 5 ? d.plane : 0;
            l2_prefetch_cells(arr[threadIdx.x], nl + off, nh + off, d.n);
          }
          double qv[UA], pc[UA];
#pragma unroll
          for (int u = 0; u < UA; ++u) {
            const int c = min(c0 + u * B, last);
            pc[u] = pcur[c];
            qv[u] = KEEP ? apply_row_diag<SYM, double>(d, A, kd[c - own.begin], pc[u],
                                                       [pcur](int cc) { return pcur[cc]; }, c)
                         : apply_row<SYM, double>(d, A, pcur, c);
          }
#pragma unroll
          for (int u = 0; u < UA; ++u) {
            const bool live = c0 + u * B < own.end;
            if (live) {
              if (KEEP)
                kq[c0 + u * B - own.begin] = qv[u];
              else
                q[c0 + u * B] = qv[u];
            }
            v1[0] = v1[0] + (live ? pc[u] * qv[u] : 0.0);
          }
        }
      } else {
        const double bt = beta;
        auto pnew = [z, pold, bt](int cc) { return z[cc] + bt * pold[cc]; };
        for (int c0 = own.begin + (int)threadIdx.x; c0 < own.end; c0 += B * UA) {
          if (PF && threadIdx.x < 8) {
            const int nl = c0 - (int)threadIdx.x + B * UA, nh = min(nl + B * UA, own.end);
            const double* arr[8] = {z, pold, aP, A.aE, A.aN, A.aT, z, pold};
            const int off = threadIdx.x >= 6 ? d.plane : 0;
            l2_prefetch_cells(arr[threadIdx.x], nl + off, nh + off, d.n);
          }
          double qv[UA], pc[UA];
#pragma unroll
          for (int u = 0; u < UA; ++u) {
            const int c = min(c0 + u * B, last);
            pc[u] = pnew(c);
            qv[u] = KEEP ? apply_row_diag<SYM, double>(d, A, kd[c - own.begin], pc[u], pnew, c)
                         : apply_row_with<SYM, double>(d, A, pc[u], pnew, c);
          }
#pragma unroll
          for (int u = 0; u < UA; ++u) {
            const bool live = c0 + u * B < own.end;
            if (live) {
              pcur[c0 + u * B] = pc[u];
              if (KEEP) {
                kq[c0 + u * B - own.begin] = qv[u];
              } else {
                q[c0 + u * B] = qv[u];
              }
            }
            v1[0] = v1[0] + (live ? pc[u] * qv[u] : 0.0);
          }
        }
      }
      if constexpr (PQS) {
        ok = g.nb <= 32 * kPerLane
                 ? group_allsum_slots(v1, g, a.ws.part + (size_t)kPqSlotOffset * g.nb)
                 : allsum<1>(v1, g, 3);
      } else {
        ok = allsum<1>(v1, g, 3);
      }
      if (!ok) break;
      const double pq = v1[0];
      if (fabs(pq) < kSmall) break;
      const double alpha = rz / pq;
      // Phase B: phi += alpha pv; r -= alpha q; r.r; z and r.z (:538-553)
      double v2[2] = {0.0, 0.0};
      for (int c0 = own.begin + (int)threadIdx.x; c0 < own.end; c0 += B * U) {
        if (PF && threadIdx.x < 5) {
          const int nl = c0 - (int)threadIdx.x + B * U, nh = min(nl + B * U, own.end);
          const double* arr[5] = {pcur, q, aP, x, r};
          l2_prefetch_cells(arr[threadIdx.x], nl, nh, d.n);
        }
        double pv[U], qv[U], dv[U], xv[U], rv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int c = min(c0 + u * B, last);
          if (KEEP) {
            const int o = c - own.begin;
            pv[u] = pcur[c];
            qv[u] = kq[o];
            dv[u] = kd[o];
            xv[u] = kx[o];
            rv[u] = kr[o];
          } else {
            pv[u] = pcur[c];
            qv[u] = q[c];
            dv[u] = aP[c];
            xv[u] = x[c];
            rv[u] = r[c];
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool live = c0 + u * B < own.end;
          const double xn = xv[u] + alpha * pv[u];
          const double rn = rv[u] - alpha * qv[u];
          const double zv = rn / guard_small(fabs(dv[u]));
          if (live) {
            const int c = c0 + u * B;
            if (KEEP) {
              kx[c - own.begin] = xn;
              kr[c - own.begin] = rn;
            } else {
              x[c] = xn;
              r[c] = rn;
            }
            z[c] = zv;
          }
          v2[0] = v2[0] + (live ? rn * rn : 0.0);
          v2[1] = v2[1] + (live ? rn * zv : 0.0);
        }
      }
      if (!(ok = allsum<2>(v2, g, 4))) break;
      residual = sqrt(v2[0]) / bnorm;
      n_iter = iter;
      if (residual < a.tol) break;
      // Once the residual is NaN the reference iterates a fixed point: the
      // next direction and every later iterate are NaN in every cell, and it
      // runs to max_iter. Produce that outcome directly.
      if (residual != residual && iter < a.max_iter) { nan_fill = true; break; }
      beta = v2[1] / guard_small(rz);
      rz = v2[1];
    }
    if (KEEP && !nan_fill) {  // the kept x back to global memory
      for (int c = own.begin + (int)threadIdx.x; c < own.end; c += B) x[c] = kx[c - own.begin];
    }
    if (nan_fill) {
      const double qnan = __longlong_as_double(0x7ff8000000000000ll);
      for (int c = own.begin + (int)threadIdx.x; c < own.end; c += B) x[c] = qnan;
      residual = qnan;
      n_iter = a.max_iter;
    }
  }
  if (g.bid == 0 && threadIdx.x == 0) {
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

// Single-system kernel variants: the register budget per thread follows the
// block size (64 at 1024 threads, 128 at 512, 255 at 256), and the larger
// budgets carry more cells per round. Every variant owns the same slices and
// visits a thread's cells in the same order, so all give the same bits for
// one launch shape.
template <int MAXB, int U, int UA, bool PF>
__global__ void __launch_bounds__(MAXB, 1) cg_f64_kernel(CgArgs a) {
  Group g;
  g.counter = a.ws.counter;
  g.err = a.ws.err;
  g.part = a.ws.part;
  g.stage = group_stage_smem();
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.timeout_ns = a.timeout_ns;
  g.epoch = 0;
  // The fence-free p.q all-reduce is for the L2-resident meshes; beyond L2
  // (PF) it measured slower (121.4 against 117.9 us per iteration at
  // 120x240x168).
  if (*a.s.asym == 0)
    cg_body<true, U, UA, PF, Group, false, !PF>(a, g);
  else
    cg_body<false, U, UA, PF, Group, false, !PF>(a, g);
}

// The same solver with the own cells' update operands kept in shared memory
// (cg_body's KEEP); the launcher sizes the dynamic shared memory for the
// largest slice.
template <int MAXB, int U, int UA>
__global__ void __launch_bounds__(MAXB, 1) cg_keep_kernel(CgArgs a) {
  extern __shared__ __align__(16) double keep_smem[];
  Group g;
  g.counter = a.ws.counter;
  g.err = a.ws.err;
  g.part = a.ws.part;
  g.stage = group_stage_smem();
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.timeout_ns = a.timeout_ns;
  g.epoch = 0;
  if (*a.s.asym == 0)
    cg_body<true, U, UA, false, Group, true, true>(a, g, keep_smem);
  else
    cg_body<false, U, UA, false, Group, true, true>(a, g, keep_smem);
}

// The same solver on a grid of thread-block clusters (cluster_red.cuh): the
// blocks, their slices and the per-cell arithmetic are those of
// cg_f64_kernel; only the all-reduces (and with them the association of the
// dot products) differ.
template <int MAXB, int U, int UA, bool PF>
__global__ void __launch_bounds__(MAXB, 1) cg_cluster_kernel(CgArgs a, double* slots) {
  ClusterGroup g = make_cluster_group(slots, a.ws.err, a.timeout_ns);
  // Every block of the cluster has started before any block addresses
  // another's shared memory.
  cluster_sync_all();
  if (*a.s.asym == 0)
    cg_body<true, U, UA, PF>(a, g);
  else
    cg_body<false, U, UA, PF>(a, g);
  // No block leaves while another block of its cluster may still address
  // its shared memory.
  cluster_sync_all();
}

// ---------------------------------------------------------------------------
// Streaming form: the same solver with every phase's operands staged in
// shared memory by bulk copies (stream_stage.cuh), a few tiles ahead of the
// threads that use them. A block walks its slice in tiles of B cells (one
// cell per thread per tile, so thread t visits the cells it visits in
// cg_body, in the same order: the dot products, the per-cell arithmetic and
// the result are bit-identical to cg_f64_kernel on the same launch). For
// the stencil phase a tile's stage holds, for cells [t0, t1):
//   the direction inputs (z and the old direction, or p in iteration 1) over
//   [t0 - nr, t1 + nr) (own cells, r and theta neighbours) and over the
//   tiles one z-plane below and above (the bottom and top neighbours),
//   aN over [t0 - nr, t1), aE over [t0 - 1, t1), aP and aT over the tile and
//   aT one plane below;
// only the theta-periodic wrap neighbours (j = 0 and j = nth - 1) are read
// from global memory directly. The update phase stages p, q, aP, x and r of
// the tile. Results go to global memory with ordinary stores, followed by a
// proxy fence so that the next phase's bulk copies (async proxy) see them
// once the all-reduce has published them. Symmetric (4-array) operators
// only; the 7-array form runs cg_body's per-thread loads in the same
// kernel.
// ---------------------------------------------------------------------------
constexpr int kMaxStages = 4;

struct StreamLayout {
  int S;      // stages
  int wc;     // capacity (doubles) of a centre window: B + 2 nr + 4
  int wb;     // capacity of a tile window: B + 4
  int stage;  // doubles per stage
};

__host__ __device__ __forceinline__ StreamLayout stream_layout(int B, int nr, int S) {
  StreamLayout L;
  L.S = S;
  L.wc = B + 2 * nr + 4;
  L.wb = B + 4;
  L.stage = 3 * L.wc + 8 * L.wb;
  return L;
}

// Stage slot offsets (doubles) of the stencil phase.
enum { kSzc, kSzd, kSzu, kSoc, kSod, kSou, kSaN, kSaE, kSaP, kSaT, kSaTd, kSlots };
__device__ __forceinline__ int slot_off(const StreamLayout& L, int k) {
  // zc, zd, zu, oc, od, ou, aN, aE, aP, aT, aTd
  const int wc = L.wc, wb = L.wb;
  switch (k) {
    case kSzc: return 0;
    case kSzd: return wc;
    case kSzu: return wc + wb;
    case kSoc: return wc + 2 * wb;
    case kSod: return 2 * wc + 2 * wb;
    case kSou: return 2 * wc + 3 * wb;
    case kSaN: return 2 * wc + 4 * wb;
    case kSaE: return 3 * wc + 4 * wb;
    case kSaP: return 3 * wc + 5 * wb;
    case kSaT: return 3 * wc + 6 * wb;
    default: return 3 * wc + 7 * wb;  // kSaTd
  }
}

struct StencilTile {
  Window zc, zd, zu, oc, od, ou, aN, aE, aP, aT, aTd;
};

// Windows of the stencil phase for tile [t0, t1) (bounds rounded out to even
// cells; the plane-shifted windows are empty where they leave the mesh).
__device__ __forceinline__ StencilTile stencil_tile(const StreamLayout& L, double* st,
                                                   const MeshDims& d, int t0, int t1) {
  StencilTile T;
  const int n = d.n, nr = d.nr, pl = d.plane;
  const int cl = even_floor(max(t0 - nr, 0)), ch = even_ceil(min(t1 + nr, n));
  int dl = even_floor(max(t0 - pl, 0)), dh = even_ceil(max(t1 - pl, 0));
  if (dh < dl) dh = dl;
  int ul = even_floor(min(t0 + pl, n)), uh = even_ceil(min(t1 + pl, n));
  if (uh < ul) uh = ul;
  const int el = even_floor(max(t0 - 1, 0)), tl = even_floor(t0), th = even_ceil(t1);
  T.zc = {st + slot_off(L, kSzc), cl, ch};
  T.zd = {st + slot_off(L, kSzd), dl, dh};
  T.zu = {st + slot_off(L, kSzu), ul, uh};
  T.oc = {st + slot_off(L, kSoc), cl, ch};
  T.od = {st + slot_off(L, kSod), dl, dh};
  T.ou = {st + slot_off(L, kSou), ul, uh};
  T.aN = {st + slot_off(L, kSaN), cl, th};
  T.aE = {st + slot_off(L, kSaE), el, th};
  T.aP = {st + slot_off(L, kSaP), tl, th};
  T.aT = {st + slot_off(L, kSaT), tl, th};
  T.aTd = {st + slot_off(L, kSaTd), dl, dh};
  return T;
}

__device__ __forceinline__ uint32_t copy_window(const Window& w, const double* src,
                                                uint64_t* bar) {
  const int cells = w.hi - w.lo;
  if (cells <= 0) return 0u;
  bulk_copy_g2s((void*)w.buf, src + w.lo, 8u * (uint32_t)cells, bar);
  return 8u * (uint32_t)cells;
}

__device__ __forceinline__ uint32_t window_bytes(const Window& w) {
  return w.hi > w.lo ? 8u * (uint32_t)(w.hi - w.lo) : 0u;
}

// Issues the stencil-phase copies of one tile (thread 0 only). `x` is the
// direction input (z, or p in iteration 1), `o` the old direction (nullptr
// in iteration 1).
__device__ void issue_stencil(const StreamLayout& L, double* st, uint64_t* bar,
                              const MeshDims& d, const SysF64& s, const double* x,
                              const double* o, int t0, int t1) {
  const StencilTile T = stencil_tile(L, st, d, t0, t1);
  uint32_t bytes = window_bytes(T.zc) + window_bytes(T.zd) + window_bytes(T.zu) +
                   window_bytes(T.aN) + window_bytes(T.aE) + window_bytes(T.aP) +
                   window_bytes(T.aT) + window_bytes(T.aTd);
  if (o) bytes += window_bytes(T.oc) + window_bytes(T.od) + window_bytes(T.ou);
  mbar_arrive_expect(bar, bytes);
  copy_window(T.zc, x, bar);
  copy_window(T.zd, x, bar);
  copy_window(T.zu, x, bar);
  if (o) {
    copy_window(T.oc, o, bar);
    copy_window(T.od, o, bar);
    copy_window(T.ou, o, bar);
  }
  copy_window(T.aN, s.aN, bar);
  copy_window(T.aE, s.aE, bar);
  copy_window(T.aP, s.aP, bar);
  copy_window(T.aT, s.aT, bar);
  copy_window(T.aTd, s.aT, bar);
}

// Update phase: p, q, aP, x, r of the tile.
__device__ __forceinline__ Window update_window(const StreamLayout& L, double* st, int k,
                                                int t0, int t1) {
  return Window{st + k * L.wb, even_floor(t0), even_ceil(t1)};
}

__device__ void issue_update(const StreamLayout& L, double* st, uint64_t* bar,
                             const SysF64& s, const double* p, int t0, int t1) {
  const Window w = update_window(L, st, 0, t0, t1);
  mbar_arrive_expect(bar, 5u * window_bytes(w));
  const double* src[5] = {p, s.q, s.aP, s.x, s.r};
#pragma unroll
  for (int k = 0; k < 5; ++k) copy_window(update_window(L, st, k, t0, t1), src[k], bar);
}

// Waits for every tile issued but not consumed (after a failed wait), so
// that no copy into this block's shared memory is in flight when it leaves.
__device__ void drain_stages(uint64_t* bars, uint32_t& par, int S, int from, int to,
                             int* err, uint64_t timeout_ns) {
  if (threadIdx.x == 0) {
    for (int t = from; t < to; ++t) {
      const int sidx = t % S;
      mbar_wait(&bars[sidx], (par >> sidx) & 1u, err, timeout_ns);
      par ^= 1u << sidx;
    }
  }
  __syncthreads();
}

__device__ void cg_stream_body(const CgArgs& a, Group& g, double* smem, uint64_t* bars,
                               const StreamLayout& L) {
  const MeshDims& d = a.d;
  const SysF64& s = a.s;
  const Slice own = own_slice(d.n, g.nb, g.bid);
  const Coefs<double> A = coefs_of<double>(s.aP, s.aE, s.aN, s.aT, s.aW, s.aS, s.aB);
  const double* __restrict__ aP = s.aP;
  const double* __restrict__ b = s.b;
  double* __restrict__ x = s.x;
  double* __restrict__ r = s.r;
  double* __restrict__ z = s.z;
  double* __restrict__ q = s.q;
  const int B = blockDim.x;
  const int S = L.S;
  const int ntile = own.end > own.begin ? (own.end - own.begin + B - 1) / B : 0;
  uint32_t par = 0;  // expected completion parity of each stage

  // Preamble (src/mod_solver_3d.f90:515-530) with per-thread loads, as cg_body.
  double v3[3] = {0.0, 0.0, 0.0};
  for (int c = own.begin + (int)threadIdx.x; c < own.end; c += B) {
    const double bv = b[c], rv = r[c];
    const double zv = rv / guard_small(fabs(aP[c]));
    s.p[c] = zv;
    v3[0] = v3[0] + bv * bv;
    v3[1] = v3[1] + rv * rv;
    v3[2] = v3[2] + rv * zv;
  }
  fence_proxy_async_global();
  bool ok = allsum<3>(v3, g, 0);
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
      const double* __restrict__ pold = (iter & 1) ? s.p2 : s.p;
      double* __restrict__ pcur = (iter & 1) ? s.p : s.p2;
      const bool first = iter == 1;
      const double* xin = first ? pcur : z;
      const double* oin = first ? nullptr : pold;
      const double bt = beta;
      // Phase A: p = z + beta p_old, q = A p, p.q (tiles of B cells).
      double v1[1] = {0.0};
      if (threadIdx.x == 0) {
        for (int t = 0; t < S && t < ntile; ++t) {
          const int t0 = own.begin + t * B;
          issue_stencil(L, smem + (size_t)t * L.stage, &bars[t], d, s, xin, oin, t0,
                        min(t0 + B, own.end));
        }
      }
      for (int t = 0; t < ntile; ++t) {
        const int sidx = t % S;
        double* st = smem + (size_t)sidx * L.stage;
        const int t0 = own.begin + t * B, t1 = min(t0 + B, own.end);
        bool w_ok = mbar_wait(&bars[sidx], (par >> sidx) & 1u, g.err, g.timeout_ns);
        par ^= 1u << sidx;
        const int c = t0 + (int)threadIdx.x;
        if (w_ok && c < t1) {
          const StencilTile T = stencil_tile(L, st, d, t0, t1);
          int i, j, k;
          cell_ijk(d, c, i, j, k);
          auto xv = [&](const Window& wz, const Window& wo, int cc) {
            return first ? wz[cc] : wz[cc] + bt * wo[cc];
          };
          auto xg = [&](int cc) { return first ? xin[cc] : xin[cc] + bt * oin[cc]; };
          const double pc = xv(T.zc, T.oc, c);
          double y = T.aP[c] * pc;
          if (i > 0) y = y - T.aE[c - 1] * xv(T.zc, T.oc, c - 1);
          if (i < d.nr - 1) y = y - T.aE[c] * xv(T.zc, T.oc, c + 1);
          if (j > 0) {
            y = y - T.aN[c - d.nr] * xv(T.zc, T.oc, c - d.nr);
          } else {
            const int cs = c + (d.nth - 1) * d.nr;
            y = y - A.aN[cs] * xg(cs);
          }
          if (j < d.nth - 1)
            y = y - T.aN[c] * xv(T.zc, T.oc, c + d.nr);
          else
            y = y - T.aN[c] * xg(c - (d.nth - 1) * d.nr);
          if (k > 0) y = y - T.aTd[c - d.plane] * xv(T.zd, T.od, c - d.plane);
          if (k < d.nz - 1) y = y - T.aT[c] * xv(T.zu, T.ou, c + d.plane);
          if (!first) pcur[c] = pc;
          q[c] = y;
          v1[0] = v1[0] + pc * y;
        }
        ok = __syncthreads_and(w_ok) != 0;
        if (!ok) {
          drain_stages(bars, par, S, t + 1, min(t + S, ntile), g.err, g.timeout_ns);
          break;
        }
        if (threadIdx.x == 0 && t + S < ntile) {
          const int n0 = own.begin + (t + S) * B;
          issue_stencil(L, st, &bars[sidx], d, s, xin, oin, n0, min(n0 + B, own.end));
        }
      }
      if (!ok) break;
      fence_proxy_async_global();
      if (!(ok = allsum<1>(v1, g, 3))) break;
      const double pq = v1[0];
      if (fabs(pq) < kSmall) break;
      const double alpha = rz / pq;
      // Phase B: phi += alpha pv; r -= alpha q; r.r; z and r.z (:538-553)
      double v2[2] = {0.0, 0.0};
      if (threadIdx.x == 0) {
        for (int t = 0; t < S && t < ntile; ++t) {
          const int t0 = own.begin + t * B;
          issue_update(L, smem + (size_t)t * L.stage, &bars[t], s, pcur, t0,
                       min(t0 + B, own.end));
        }
      }
      for (int t = 0; t < ntile; ++t) {
        const int sidx = t % S;
        double* st = smem + (size_t)sidx * L.stage;
        const int t0 = own.begin + t * B, t1 = min(t0 + B, own.end);
        bool w_ok = mbar_wait(&bars[sidx], (par >> sidx) & 1u, g.err, g.timeout_ns);
        par ^= 1u << sidx;
        const int c = t0 + (int)threadIdx.x;
        if (w_ok && c < t1) {
          const double pv = update_window(L, st, 0, t0, t1)[c];
          const double qv = update_window(L, st, 1, t0, t1)[c];
          const double dv = update_window(L, st, 2, t0, t1)[c];
          const double xv0 = update_window(L, st, 3, t0, t1)[c];
          const double rv = update_window(L, st, 4, t0, t1)[c];
          const double xn = xv0 + alpha * pv;
          const double rn = rv - alpha * qv;
          const double zv = rn / guard_small(fabs(dv));
          x[c] = xn;
          r[c] = rn;
          z[c] = zv;
          v2[0] = v2[0] + rn * rn;
          v2[1] = v2[1] + rn * zv;
        }
        ok = __syncthreads_and(w_ok) != 0;
        if (!ok) {
          drain_stages(bars, par, S, t + 1, min(t + S, ntile), g.err, g.timeout_ns);
          break;
        }
        if (threadIdx.x == 0 && t + S < ntile) {
          const int n0 = own.begin + (t + S) * B;
          issue_update(L, st, &bars[sidx], s, pcur, n0, min(n0 + B, own.end));
        }
      }
      if (!ok) break;
      fence_proxy_async_global();
      if (!(ok = allsum<2>(v2, g, 4))) break;
      residual = sqrt(v2[0]) / bnorm;
      n_iter = iter;
      if (residual < a.tol) break;
      if (residual != residual && iter < a.max_iter) { nan_fill = true; break; }
      beta = v2[1] / guard_small(rz);
      rz = v2[1];
    }
    if (nan_fill) {
      const double qnan = __longlong_as_double(0x7ff8000000000000ll);
      for (int c = own.begin + (int)threadIdx.x; c < own.end; c += B) x[c] = qnan;
      residual = qnan;
      n_iter = a.max_iter;
    }
  }
  if (g.bid == 0 && threadIdx.x == 0) {
    SolveResult* res = a.ws.result;
    const int err = ld_volatile_i32(a.ws.err);
    res->status = err != 0 ? err : (isfinite(residual) ? EAF_OK : EAF_ENONFINITE);
    res->n_iter = n_iter;
    res->n_outer = 0;
    res->sym = 1;
    res->residual = residual;
    res->bnorm = bnorm;
  }
}

template <int MAXB, int U, int UA>
__global__ void __launch_bounds__(MAXB, 1) cg_stream_kernel(CgArgs a, int stages) {
  extern __shared__ __align__(128) double stream_smem[];
  __shared__ __align__(8) uint64_t bars[kMaxStages];
  Group g;
  g.counter = a.ws.counter;
  g.err = a.ws.err;
  g.part = a.ws.part;
  g.stage = group_stage_smem();
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.timeout_ns = a.timeout_ns;
  g.epoch = 0;
  if (*a.s.asym != 0) {
    cg_body<false, U, UA, false>(a, g);
    return;
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < stages; ++k) mbar_init(&bars[k], 1);
    mbar_fence_init();
  }
  __syncthreads();
  cg_stream_body(a, g, stream_smem, bars, stream_layout(blockDim.x, a.d.nr, stages));
}

__global__ void fill_marker_kernel(double* p, int n) {
  const double marker = __longlong_as_double((long long)kSlotMarker);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = marker;
}

// ---------------------------------------------------------------------------
// Single-reduction form (Chronopoulos and Gear, J. Comput. Appl. Math. 25,
// 1989): the same preconditioned CG with its recurrences rearranged so that an
// iteration is ONE phase closed by ONE group all-reduce of three sums:
//   own cells: u = r dinv, p = u + beta p, s = w + beta s,
//   x += alpha p, r' = r - alpha s, u' = r' dinv, w' = A u'
//   (dinv = 1 / max(|aP|, SMALL), stored by the preamble: the Jacobi step is
//   a multiply here, not the reference's division)
//   (the six neighbours' u' formed here from their stored r, w and s, final
//   since the last barrier), partial r'.u', w'.u', r'.r'  -> all-reduce
// then beta = gamma / max(gamma_prev, SMALL), p.q = delta - beta gamma /
// alpha_prev, alpha = gamma / p.q, evaluated by every block. r, w and s are
// double-buffered (neighbours read the old ones while owners write the new);
// p and x are own-cell only. Iteration 1 takes p = u and s = w exactly. The
// exit tests, the preconditioner, the stencil's expression order and the NaN
// outcome are the reference's; the partial table alternates between two slot
// sets so that a block's next partials never overwrite ones a slower block
// is still folding. Parity: bit for bit with the oracle's restatement of
// this form in the kernels' association (eaf_oracle_cg1); against the
// reference's recurrences, the same residual ball.
template <bool SYM, int U>
__device__ void cg1_body(const CgArgs& a, Group& g) {
  const MeshDims& d = a.d;
  const SysF64& s = a.s;
  const Slice own = own_slice(d.n, g.nb, g.bid);
  const Coefs<double> A = coefs_of<double>(s.aP, s.aE, s.aN, s.aT, s.aW, s.aS, s.aB);
  const double* __restrict__ aP = s.aP;
  const double* __restrict__ b = s.b;
  double* __restrict__ x = s.x;
  double* __restrict__ p = s.p;
  const int B = blockDim.x;
  const int last = own.end - 1;

  // Preamble: dinv = 1 / max(|aP|, SMALL) stored, u0 = r0 * dinv,
  // w0 = A u0; b.b, r.r, r.u, w.u.
  double v4[4] = {0.0, 0.0, 0.0, 0.0};
  double* __restrict__ dinv = s.dinv;
  {
    const double* __restrict__ r0 = s.r;
    double* __restrict__ w0 = s.q;
    auto u0 = [r0, aP](int cc) { return r0[cc] * (1.0 / guard_small(fabs(aP[cc]))); };
    for (int c0 = own.begin + (int)threadIdx.x; c0 < own.end; c0 += B * U) {
      double bv[U], rv[U], uv[U], wv[U], iv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int c = min(c0 + u * B, last);
        bv[u] = b[c];
        rv[u] = r0[c];
        iv[u] = 1.0 / guard_small(fabs(aP[c]));
        uv[u] = rv[u] * iv[u];
        wv[u] = apply_row_with<SYM, double>(d, A, uv[u], u0, c);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool live = c0 + u * B < own.end;
        if (live) {
          w0[c0 + u * B] = wv[u];
          dinv[c0 + u * B] = iv[u];
        }
        v4[0] = v4[0] + (live ? bv[u] * bv[u] : 0.0);
        v4[1] = v4[1] + (live ? rv[u] * rv[u] : 0.0);
        v4[2] = v4[2] + (live ? rv[u] * uv[u] : 0.0);
        v4[3] = v4[3] + (live ? wv[u] * uv[u] : 0.0);
      }
    }
  }
  bool ok = group_allsum<4>(v4, g, 0);
  const double bnorm = sqrt(v4[0]);
  double residual = 0.0;
  int n_iter = 0;
  bool nan_fill = false;
  if (ok && !(bnorm < kSmall)) {
    double gam = v4[2], dlt = v4[3], gam_prev = 0.0, alpha_prev = 0.0;
    residual = sqrt(v4[1]) / bnorm;
    if (residual != residual && a.max_iter >= 1) nan_fill = true;
    for (int iter = 1; iter <= a.max_iter && !nan_fill; ++iter) {
      const bool first = iter == 1;
      double beta = 0.0, den;
      if (first) {
        den = dlt;
      } else {
        beta = gam / guard_small(gam_prev);
        den = dlt - beta * gam / alpha_prev;
      }
      if (fabs(den) < kSmall) break;
      const double alpha = gam / den;
      // buffers: r in (r, z), w in (q, p2), s in (s0, s1); odd iterations
      // read the first of each pair
      const bool odd = (iter & 1) != 0;
      const double* __restrict__ rc = odd ? s.r : s.z;
      const double* __restrict__ wc = odd ? s.q : s.p2;
      const double* __restrict__ sc = odd ? s.s0 : s.s1;
      double* __restrict__ rn = odd ? s.z : s.r;
      double* __restrict__ wn = odd ? s.p2 : s.q;
      double* __restrict__ sn = odd ? s.s1 : s.s0;
      // a neighbour's new preconditioned residual, from its stored values
      auto unew = [rc, wc, sc, dinv, first, alpha, beta](int cc) {
        const double sv = first ? wc[cc] : wc[cc] + beta * sc[cc];
        const double rv = rc[cc] - alpha * sv;
        return rv * dinv[cc];
      };
      double v3[3] = {0.0, 0.0, 0.0};
      for (int c0 = own.begin + (int)threadIdx.x; c0 < own.end; c0 += B * U) {
        double rv[U], wv[U], sv[U], pv[U], xv[U], dv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int c = min(c0 + u * B, last);
          rv[u] = rc[c];
          wv[u] = wc[c];
          sv[u] = first ? 0.0 : sc[c];
          pv[u] = first ? 0.0 : p[c];
          xv[u] = x[c];
          dv[u] = dinv[c];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int c = min(c0 + u * B, last);
          const bool live = c0 + u * B < own.end;
          const double g0 = dv[u];
          const double uo = rv[u] * g0;
          const double pn = first ? uo : uo + beta * pv[u];
          const double snv = first ? wv[u] : wv[u] + beta * sv[u];
          const double xn = xv[u] + alpha * pn;
          const double rnv = rv[u] - alpha * snv;
          const double un = rnv * g0;
          const double wnv = apply_row_with<SYM, double>(d, A, un, unew, c);
          if (live) {
            p[c] = pn;
            sn[c] = snv;
            x[c] = xn;
            rn[c] = rnv;
            wn[c] = wnv;
          }
          v3[0] = v3[0] + (live ? rnv * un : 0.0);
          v3[1] = v3[1] + (live ? wnv * un : 0.0);
          v3[2] = v3[2] + (live ? rnv * rnv : 0.0);
        }
      }
      if (!(ok = group_allsum<3>(v3, g, (iter & 1) ? 4 : 0))) break;
      gam_prev = gam;
      alpha_prev = alpha;
      gam = v3[0];
      dlt = v3[1];
      residual = sqrt(v3[2]) / bnorm;
      n_iter = iter;
      if (residual < a.tol) break;
      if (residual != residual && iter < a.max_iter) { nan_fill = true; break; }
    }
    if (nan_fill) {
      const double qnan = __longlong_as_double(0x7ff8000000000000ll);
      for (int c = own.begin + (int)threadIdx.x; c < own.end; c += B) x[c] = qnan;
      residual = qnan;
      n_iter = a.max_iter;
    }
  }
  if (g.bid == 0 && threadIdx.x == 0) {
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

template <int MAXB, int U>
__global__ void __launch_bounds__(MAXB, 1) cg1_f64_kernel(CgArgs a) {
  Group g;
  g.counter = a.ws.counter;
  g.err = a.ws.err;
  g.part = a.ws.part;
  g.stage = group_stage_smem();
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.timeout_ns = a.timeout_ns;
  g.epoch = 0;
  if (*a.s.asym == 0)
    cg1_body<true, U>(a, g);
  else
    cg1_body<false, U>(a, g);
}

// ---------------------------------------------------------------------------
// Batched launch (see BatchTables): the same solver body per system, on the
// lane's blocks with the lane's barrier counter and partial table.
// ---------------------------------------------------------------------------
struct BatchF64Args {
  BatchTables t;
  int max_iter;
  double tol;
  uint64_t timeout_ns;
};

// Blocks of kBatchBlock threads, two per SM (64 registers a thread): a batch
// is throughput-bound over many small systems, so co-resident lanes count
// for more than per-lane speed (the 128-register form with one block per SM
// ran the 96-system mix 12 % slower).
__global__ void __launch_bounds__(kBatchBlock, 2) batch_f64_kernel(BatchF64Args a) {
  const int lane = a.t.lane_of_block[blockIdx.x];
  const int first = a.t.lane_first_block[lane];
  Group g;
  g.counter = a.t.counters + (size_t)lane * kCounterStride;
  g.err = a.t.err;
  g.part = a.t.parts + (size_t)8 * first;
  g.stage = group_stage_smem();
  g.nb = a.t.lane_width[lane];
  g.bid = blockIdx.x - first;
  g.timeout_ns = a.timeout_ns;
  g.epoch = 0;
  for (int qi = a.t.lane_q_begin[lane]; qi < a.t.lane_q_begin[lane + 1]; ++qi) {
    if (ld_volatile_i32(a.t.err) != 0) break;
    const BatchSys& bs = a.t.sys[a.t.queue[qi]];
    CgArgs ca;
    ca.d = bs.d;
    ca.s = bs.s;
    ca.ws.part = g.part;
    ca.ws.counter = g.counter;
    ca.ws.err = a.t.err;
    ca.ws.result = bs.result;
    ca.max_iter = a.max_iter;
    ca.tol = a.tol;
    ca.timeout_ns = a.timeout_ns;
    // The lanes keep the counter form for p.q: many lanes polling without
    // the release measured slower (157.0 against 161.7 solves/s on the
    // 96-system mix).
    if (*bs.s.asym == 0)
      cg_body<true, 2, 1, false, Group>(ca, g);
    else
      cg_body<false, 2, 1, false, Group>(ca, g);
  }
}

// ---------------------------------------------------------------------------
// pack / unpack
// ---------------------------------------------------------------------------
struct PackArgs {
  MeshDims d;
  HaloInputs in;
  SysF64 s;
  long long hy, hz;  // halo strides of j and k
};

__global__ void pack_f64_kernel(PackArgs a) {
  const MeshDims& d = a.d;
  const HaloInputs& in = a.in;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_ijk(d, c, i, j, k);
    const long long h = (long long)(i + 2) + a.hy * (j + 2) + a.hz * (k + 2);
    const long long hs = j > 0 ? h - a.hy : h + (long long)(d.nth - 1) * a.hy;
    const long long hn = j < d.nth - 1 ? h + a.hy : h - (long long)(d.nth - 1) * a.hy;
    const double aW = in.aW[h], aE = in.aE[h], aS = in.aS[h], aN = in.aN[h];
    const double aB = in.aB[h], aT = in.aT[h], aP = in.aP[h], su = in.Su[h];
    a.s.aP[c] = aP;
    a.s.aE[c] = aE;
    a.s.aN[c] = aN;
    a.s.aT[c] = aT;
    a.s.aW[c] = aW;
    a.s.aS[c] = aS;
    a.s.aB[c] = aB;
    a.s.b[c] = su;
    // Symmetric-form test: every link equals its partner's, wall links are
    // zero (compared by value; a NaN link selects the general form).
    const bool sym = (aW == (i > 0 ? in.aE[h - 1] : 0.0)) &&
                     (i < d.nr - 1 || aE == 0.0) && (aS == in.aN[hs]) &&
                     (aB == (k > 0 ? in.aT[h - a.hz] : 0.0)) &&
                     (k < d.nz - 1 || aT == 0.0);
    if (!sym) atomicOr(a.s.asym, 1);
    // r = Su - A*phi exactly as the reference's first matvec
    // (src/mod_solver_3d.f90:510-513): theta-wrapped interior neighbours,
    // r/z halo cells of phi as given.
    const double xc = in.phi[h];
    const double y = aP * xc - aW * in.phi[h - 1] - aE * in.phi[h + 1] -
                     aS * in.phi[hs] - aN * in.phi[hn] - aB * in.phi[h - a.hz] -
                     aT * in.phi[h + a.hz];
    a.s.x[c] = xc;
    a.s.r[c] = su - y;
  }
}

struct UnpackArgs {
  MeshDims d;
  const double* x;
  double* phi;
  int hy;            // nr + 4
  int hj;            // nth + 4
  FastDiv fd_hy, fd_hj;
  long long total;   // (nr+4)(nth+4)(nz+4)
};

// Source column of a theta-halo column j in the reference's sequential copy
// x(:,0,:)=x(:,nth,:); x(:,-1,:)=x(:,nth-1,:); x(:,nth+1,:)=x(:,1,:);
// x(:,nth+2,:)=x(:,2,:) (src/mod_mpi_topology.f90:303-311), resolved to an
// interior column (only differs from the plain rule when nth < 2).
__device__ __forceinline__ int theta_source(int j, int nth) {
  if (j == 0) return nth;
  if (j == -1) return nth - 1 >= 1 ? nth - 1 : nth;
  if (j == nth + 1) return 1;
  return 2 <= nth ? 2 : 1;  // j == nth + 2
}

__global__ void unpack_f64_kernel(UnpackArgs a) {
  const MeshDims& d = a.d;
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < a.total;
       h += (long long)gridDim.x * blockDim.x) {
    // halo coordinates -> Fortran indices
    const uint32_t t = a.fd_hy.div((uint32_t)h);
    const int i = (int)(h - (long long)t * a.hy) - 1;
    const uint32_t kk = a.fd_hj.div(t);
    const int j = (int)(t - kk * a.hj) - 1;
    const int k = (int)kk - 1;
    const bool iin = i >= 1 && i <= d.nr, kin = k >= 1 && k <= d.nz;
    const bool jin = j >= 1 && j <= d.nth;
    if (jin) {
      if (iin && kin) a.phi[h] = a.x[(i - 1) + d.nr * ((j - 1) + d.nth * (k - 1))];
    } else {
      const int js = theta_source(j, d.nth);
      if (iin && kin)
        a.phi[h] = a.x[(i - 1) + d.nr * ((js - 1) + d.nth * (k - 1))];
      else
        a.phi[h] = a.phi[h + (long long)(js - j) * a.hy];
    }
  }
}

}  // namespace

cudaError_t launch_pack_f64(const MeshDims& d, const HaloInputs& in, const SysF64& s,
                            cudaStream_t st) {
  PackArgs a;
  a.d = d;
  a.in = in;
  a.s = s;
  a.hy = d.nr + 4;
  a.hz = (long long)(d.nr + 4) * (d.nth + 4);
  (void)cudaGetLastError();  // report this launch's error, not an older one
  cudaError_t e = cudaMemsetAsync(s.asym, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int block = 256;
  int grid = (d.n + block - 1) / block;
  if (grid > 148 * 16) grid = 148 * 16;
  pack_f64_kernel<<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_unpack_f64(const MeshDims& d, const double* x, double* phi,
                              cudaStream_t st) {
  UnpackArgs a;
  a.d = d;
  a.x = x;
  a.phi = phi;
  a.hy = d.nr + 4;
  a.hj = d.nth + 4;
  a.fd_hy = FastDiv((uint32_t)a.hy);
  a.fd_hj = FastDiv((uint32_t)a.hj);
  a.total = (long long)(d.nr + 4) * (d.nth + 4) * (d.nz + 4);
  (void)cudaGetLastError();  // report this launch's error, not an older one
  const int block = 256;
  long long g = (a.total + block - 1) / block;
  int grid = (int)(g > 148 * 16 ? 148 * 16 : g);
  unpack_f64_kernel<<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

// Self-test of group_allsum_slots' bounded waits. mode 0: two blocks of a
// group declared with three members (the third never arrives, so the count
// never completes); mode 1: one block of a group of two, the count preset to
// one arrival, the other block's slot left holding the marker (its partial
// never comes). Every wait expires and the kernel reports EAF_ETIMEOUT.
__global__ void allreduce_selftest_kernel(GroupWs ws, uint64_t timeout_ns, int mode) {
  Group g;
  g.counter = ws.counter;
  g.err = ws.err;
  g.part = ws.part;
  g.stage = group_stage_smem();
  g.nb = mode == 0 ? 3 : 2;
  g.bid = blockIdx.x;
  g.timeout_ns = timeout_ns;
  g.epoch = 0;
  double v[1] = {1.0};
  group_allsum_slots(v, g, ws.part);
}

cudaError_t launch_allreduce_selftest(const GroupWs& ws, uint64_t timeout_ns, int mode,
                                      cudaStream_t st) {
  if (mode != 0 && mode != 1) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess && mode == 1) {
    const unsigned long long one = 1;
    e = cudaMemcpyAsync(ws.counter, &one, sizeof(one), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // `one` lives on this frame
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  fill_marker_kernel<<<1, 32, 0, st>>>(ws.part, 16);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  void* args[] = {(void*)&ws, (void*)&timeout_ns, (void*)&mode};
  return cudaLaunchCooperativeKernel((const void*)allreduce_selftest_kernel,
                                     dim3(mode == 0 ? 2 : 1), dim3(64), args, 0, st);
}

// The two p.q slot sets of a flat launch of `grid` blocks, filled with the
// empty-slot marker (group_allsum_slots).
static cudaError_t fill_pq_slots(const GroupWs& ws, int grid, cudaStream_t st) {
  // (harmless where the kernel keeps the counter form for p.q)
  if (grid <= 1 || grid > 32 * kPerLane) return cudaSuccess;
  fill_marker_kernel<<<1, 320, 0, st>>>(ws.part + (size_t)kPqSlotOffset * grid, 2 * grid);
  return cudaGetLastError();
}

cudaError_t launch_cg_f64(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                          int max_iter, double tol, uint64_t timeout_ns, int grid,
                          int block, cudaStream_t st) {
  CgArgs a;
  a.d = d;
  a.s = s;
  a.ws = ws;
  a.max_iter = max_iter;
  a.tol = tol;
  a.timeout_ns = timeout_ns;
  cudaError_t e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = fill_pq_slots(ws, grid, st);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel(cg_f64_kernel_ptr(block, d.n), dim3(grid),
                                     dim3(block), args, 0, st);
}

cudaError_t launch_cg1_f64(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                           int max_iter, double tol, uint64_t timeout_ns, int grid,
                           int block, cudaStream_t st) {
  if (!s.s0 || !s.s1) return cudaErrorInvalidValue;
  CgArgs a;
  a.d = d;
  a.s = s;
  a.ws = ws;
  a.max_iter = max_iter;
  a.tol = tol;
  a.timeout_ns = timeout_ns;
  cudaError_t e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel(cg1_f64_kernel_ptr(block), dim3(grid), dim3(block), args,
                                     0, st);
}

const void* cg1_f64_kernel_ptr(int block) {
  if (block <= 256) return (const void*)cg1_f64_kernel<256, 4>;
  if (block <= 512) return (const void*)cg1_f64_kernel<512, 2>;
  return (const void*)cg1_f64_kernel<1024, 1>;
}

const void* cg_cluster_kernel_ptr(int block, long long n) {
  if (block <= 256) return (const void*)cg_cluster_kernel<256, 4, 4, false>;
  if (block <= 512) return (const void*)cg_cluster_kernel<512, 4, 2, false>;
  if (l2_prefetch_pays(n)) return (const void*)cg_cluster_kernel<1024, 2, 1, true>;
  return (const void*)cg_cluster_kernel<1024, 2, 1, false>;
}

static cudaLaunchConfig_t cluster_config(int grid, int block, int cluster, cudaStream_t st,
                                         cudaLaunchAttribute* attr, bool cooperative) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeCooperative;
  attr[1].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = cooperative ? 2 : 1;
  return cfg;
}

static cudaError_t allow_cluster_size(const void* k, int cluster) {
  if (cluster <= 8) return cudaSuccess;
  return cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

int max_active_clusters(int block, long long n, int cluster) {
  if (cluster < 1 || cluster > kMaxClusterSize) return 0;
  const void* k = cg_cluster_kernel_ptr(block, n);
  if (allow_cluster_size(k, cluster) != cudaSuccess) return 0;
  cudaLaunchAttribute attr[2];
  cudaLaunchConfig_t cfg = cluster_config(cluster, block, cluster, nullptr, attr, false);
  int count = 0;
  if (cudaOccupancyMaxActiveClusters(&count, k, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return count;
}

cudaError_t launch_cg_f64_cluster(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                                  double* slots, size_t slot_doubles, int max_iter,
                                  double tol, uint64_t timeout_ns, int grid, int block,
                                  int cluster, cudaStream_t st) {
  if (cluster < 1 || cluster > kMaxClusterSize || grid % cluster != 0 ||
      grid / cluster > kMaxClusters || cluster_slot_doubles(grid / cluster) > slot_doubles)
    return cudaErrorInvalidValue;
  CgArgs a;
  a.d = d;
  a.s = s;
  a.ws = ws;
  a.max_iter = max_iter;
  a.tol = tol;
  a.timeout_ns = timeout_ns;
  const void* k = cg_cluster_kernel_ptr(block, d.n);
  cudaError_t e = allow_cluster_size(k, cluster);
  if (e != cudaSuccess) return e;
  (void)cudaGetLastError();  // report this launch's error, not an older one
  const int nslots = (int)cluster_slot_doubles(grid / cluster);
  fill_marker_kernel<<<(nslots + 255) / 256, 256, 0, st>>>(slots, nslots);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  void* args[] = {&a, &slots};
  cudaLaunchAttribute attr[2];
  cudaLaunchConfig_t cfg = cluster_config(grid, block, cluster, st, attr, true);
  e = cudaLaunchKernelExC(&cfg, k, args);
  if (e != cudaSuccess) {
    // Without the cooperative attribute the launch is the same; every wait
    // in the kernel is bounded, so blocks that were not co-scheduled end in
    // EAF_ETIMEOUT rather than a hang.
    (void)cudaGetLastError();
    cfg = cluster_config(grid, block, cluster, st, attr, false);
    e = cudaLaunchKernelExC(&cfg, k, args);
  }
  return e;
}

static const void* cg_stream_kernel_ptr(int block) {
  if (block <= 256) return (const void*)cg_stream_kernel<256, 4, 4>;
  if (block <= 512) return (const void*)cg_stream_kernel<512, 4, 2>;
  return (const void*)cg_stream_kernel<1024, 2, 1>;
}

// Stages of the streaming kernel for blocks of `block` threads on a mesh with
// nr cells per r row (0 if fewer than two fit in shared memory).
int stream_stages(int block, int nr) {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
      cudaSuccess)
    return 0;
  const long long stage = (long long)stream_layout(block, nr, 2).stage * 8;
  const long long avail = (long long)optin - 16 * 1024;  // static shared memory and slack
  long long S = avail / stage;
  if (S > kMaxStages) S = kMaxStages;
  return S >= 2 ? (int)S : 0;
}

int stream_max_coresident(int block, int nr, int sms) {
  const int S = stream_stages(block, nr);
  if (S < 2) return 0;
  const void* k = cg_stream_kernel_ptr(block);
  const size_t smem = (size_t)stream_layout(block, nr, S).stage * 8 * S;
  std::lock_guard<std::mutex> attr_lock(launch_attr_mutex());
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem) != cudaSuccess)
    return 0;
  return per_sm * sms;
}

cudaError_t launch_cg_f64_stream(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                                 int max_iter, double tol, uint64_t timeout_ns, int grid,
                                 int block, cudaStream_t st) {
  const int S = stream_stages(block, d.nr);
  if (S < 2 || block % 32 != 0) return cudaErrorInvalidValue;
  CgArgs a;
  a.d = d;
  a.s = s;
  a.ws = ws;
  a.max_iter = max_iter;
  a.tol = tol;
  a.timeout_ns = timeout_ns;
  const void* k = cg_stream_kernel_ptr(block);
  const size_t smem = (size_t)stream_layout(block, d.nr, S).stage * 8 * S;
  std::lock_guard<std::mutex> attr_lock(launch_attr_mutex());
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  int stages = S;
  void* args[] = {&a, &stages};
  return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(block), args, smem, st);
}

// The variant for blocks of `block` threads over slices of `chunk` cells.
// Where a 512-thread block's threads own at most two cells each, rounds of
// two cells in the update phase leave no dead lanes to compute (35x70x50 on
// 148 blocks: 6.7 against 7.0 us per iteration); every variant visits a
// thread's cells in the same order, so all give the same bits.
static const void* cg_keep_kernel_ptr(int block, long long chunk) {
  if (block <= 256) return (const void*)cg_keep_kernel<256, 4, 4>;
  if (block <= 512)
    return (chunk + block - 1) / block <= 2 ? (const void*)cg_keep_kernel<512, 2, 2>
                                            : (const void*)cg_keep_kernel<512, 4, 2>;
  return (const void*)cg_keep_kernel<1024, 2, 1>;
}

size_t keep_smem_bytes(long long n, int grid) {
  const long long chunk = (n + grid - 1) / grid;
  return (size_t)chunk * kKeepArrays * sizeof(double);
}

int keep_max_coresident(int block, long long n, int grid, int sms) {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
          cudaSuccess)
    return 0;
  const size_t smem = keep_smem_bytes(n, grid);
  if (smem + 8 * 1024 > (size_t)optin) return 0;  // static shared memory and slack
  const void* k = cg_keep_kernel_ptr(block, (n + grid - 1) / grid);
  std::lock_guard<std::mutex> attr_lock(launch_attr_mutex());
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return per_sm * sms;
}

cudaError_t launch_cg_f64_keep(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                               int max_iter, double tol, uint64_t timeout_ns, int grid,
                               int block, cudaStream_t st) {
  CgArgs a;
  a.d = d;
  a.s = s;
  a.ws = ws;
  a.max_iter = max_iter;
  a.tol = tol;
  a.timeout_ns = timeout_ns;
  const void* k = cg_keep_kernel_ptr(block, (d.n + grid - 1) / grid);
  const size_t smem = keep_smem_bytes(d.n, grid);
  std::lock_guard<std::mutex> attr_lock(launch_attr_mutex());
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = fill_pq_slots(ws, grid, st);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(block), args, smem, st);
}

bool l2_prefetch_pays(long long n) { return (double)n * 128.0 > 96.0e6; }

const void* cg_f64_kernel_ptr(int block, long long n) {
  if (block <= 256) return (const void*)cg_f64_kernel<256, 4, 4, false>;
  if (block <= 512) return (const void*)cg_f64_kernel<512, 4, 2, false>;
  if (l2_prefetch_pays(n)) return (const void*)cg_f64_kernel<1024, 2, 1, true>;
  return (const void*)cg_f64_kernel<1024, 2, 1, false>;
}


cudaError_t launch_batch_f64(const BatchTables& t, int grid, int block, int max_iter,
                             double tol, uint64_t timeout_ns, cudaStream_t st) {
  BatchF64Args a;
  a.t = t;
  a.max_iter = max_iter;
  a.tol = tol;
  a.timeout_ns = timeout_ns;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, batch_f64_kernel, a);
}

const void* batch_f64_kernel_ptr() { return (const void*)batch_f64_kernel; }



}  // namespace eaf
