// Mixed-precision pressure-correction CG: FP32 Jacobi-PCG inner iterations
// inside an FP64 iterative-refinement loop, one persistent cooperative
// launch per solve. No reference counterpart; it solves the same system as
// cg_3d_mpi (src/mod_solver_3d.f90:485-620) behind the same array contract.
//
// FP64 is kept for exactly four things: the solution x, the refinement
// residual r = Su - A x (FP64 coefficients), its norm (the convergence test
// ||Su - A x|| / ||Su|| < tol) and therefore the pinned reference cell, whose
// identity row stays exact. Everything the inner iterations touch is FP32:
// the coefficient copies (made once per solve), the residual estimate rs,
// the direction p, q = A p and the correction e; their dot products are
// accumulated per thread and per warp tree in FP32 (block partials are
// folded across blocks in FP64).
//
// Refinement policy (classic iterative refinement): each outer step runs a
// fresh FP32 CG on A e = r, from e = 0, until its recurred residual has
// dropped by `inner_tol` (or below tol * ||Su||, or max_inner iterations,
// or breakdown); x += e in FP64; r = Su - A x is recomputed with the FP64
// operator; stop when ||r|| / ||Su|| < tol or after max_outer steps. The
// inner CG restarts at every step: on these operators FP32 directions kept
// across a residual replacement lose conjugacy and stall the solve.
#include <math.h>

#include "cg_kernels.h"
#include "stencil.cuh"

namespace eaf {
namespace {

constexpr int kUnroll = 2;
constexpr int kMaxBlock = 1024;

struct MixArgs {
  MeshDims d;
  SysF64 s;
  SysF32 f;
  GroupWs ws;
  int max_outer, max_inner;
  double tol, inner_tol;
  uint64_t timeout_ns;
  double* trace;  // per refinement step: inner iterations, inner reduction, residual
};

template <bool SYM>
__device__ void mixed_body(const MixArgs& a, Group& g) {
  const MeshDims& d = a.d;
  const SysF64& s = a.s;
  const SysF32& f = a.f;
  const Slice own = own_slice(d.n, g.nb, g.bid);
  const Coefs<double> A64 = coefs_of<double>(s.aP, s.aE, s.aN, s.aT, s.aW, s.aS, s.aB);
  const Coefs<float> A32 = coefs_of<float>(f.aP, f.aE, f.aN, f.aT, f.aW, f.aS, f.aB);
  const double* __restrict__ b = s.b;
  double* __restrict__ x = s.x;
  const float* __restrict__ dP = f.aP;
  float* __restrict__ rs = f.r;
  float* __restrict__ zs = f.z;
  float* __restrict__ q = f.q;
  float* __restrict__ e = f.e;
#define EAF_OWN_CELLS(...) EAF_FOR_OWN(own, kUnroll, c, __VA_ARGS__)

  // Setup: FP32 coefficient copies (once per solve).
  EAF_OWN_CELLS({
    f.aP[c] = (float)s.aP[c];
    f.aE[c] = (float)s.aE[c];
    f.aN[c] = (float)s.aN[c];
    f.aT[c] = (float)s.aT[c];
    if (!SYM) {
      f.aW[c] = (float)s.aW[c];
      f.aS[c] = (float)s.aS[c];
      f.aB[c] = (float)s.aB[c];
    }
  })
  // ||Su||^2 and the first outer residual r = Su - A phi (from pack).
  double v64[2] = {0.0, 0.0};
  EAF_OWN_CELLS({
    const double bv = b[c], rv = s.r[c];
    v64[0] = v64[0] + bv * bv;
    v64[1] = v64[1] + rv * rv;
  })
  bool ok = group_allsum<2>(v64, g, 0);
  const double bnorm = sqrt(v64[0]);
  double residual = 0.0;
  int total_it = 0, outer = 0;
  if (ok && !(bnorm < kSmall)) {
    residual = sqrt(v64[1]) / bnorm;
    while (residual >= a.tol && outer < a.max_outer) {  // NaN leaves too
      // Restart of the inner CG on A e = r (FP32): rs = r, z = rs/d,
      // p = z, e = 0. The first time r is pack's residual; afterwards the
      // refinement below has just written it to s.r.
      float w32[2] = {0.f, 0.f};
      float* __restrict__ p0 = f.p;
      EAF_OWN_CELLS({
        const float r32 = (float)s.r[c];
        const float z = r32 / guard_small(fabsf(dP[c]));
        rs[c] = r32;
        zs[c] = z;
        p0[c] = z;
        e[c] = 0.f;
        w32[0] = w32[0] + r32 * r32;
        w32[1] = w32[1] + r32 * z;
      })
      if (!(ok = group_allsum<2>(w32, g, 2))) break;
      float rz = w32[1];
      const float seg_start = sqrtf(w32[0]);
      const int it_before = total_it;
      float seg_end = seg_start;
      const float stop_abs = fmaxf((float)a.inner_tol * seg_start, (float)(a.tol * bnorm));
      float beta = 0.f;
      // Inner FP32 Jacobi-PCG, two group reductions per iteration (the
      // direction update is fused into the stencil phase as in the FP64
      // kernel, with the direction double-buffered in f.p / f.p2).
      for (int k = 1; k <= a.max_inner; ++k) {
        const float* __restrict__ pold = (k & 1) ? f.p2 : f.p;
        float* __restrict__ pcur = (k & 1) ? f.p : f.p2;
        float v1[1] = {0.f};
        if (k == 1) {
          EAF_OWN_CELLS({
            const float qv = apply_row<SYM, float>(d, A32, pcur, c);
            q[c] = qv;
            v1[0] = v1[0] + pcur[c] * qv;
          })
        } else {
          const float bt = beta;
          auto pnew = [zs, pold, bt](int cc) { return zs[cc] + bt * pold[cc]; };
          EAF_OWN_CELLS({
            const float pc = pnew(c);
            const float qv = apply_row_with<SYM, float>(d, A32, pc, pnew, c);
            pcur[c] = pc;
            q[c] = qv;
            v1[0] = v1[0] + pc * qv;
          })
        }
        if (!(ok = group_allsum<1>(v1, g, 4))) break;
        const float pq = v1[0];
        if (!(fabsf(pq) >= 1.0e-30f)) break;  // breakdown (or NaN)
        const float alpha = rz / pq;
        float v2[2] = {0.f, 0.f};
        EAF_OWN_CELLS({
          e[c] = e[c] + alpha * pcur[c];
          const float rv = rs[c] - alpha * q[c];
          rs[c] = rv;
          const float z = rv / guard_small(fabsf(dP[c]));
          zs[c] = z;
          v2[0] = v2[0] + rv * rv;
          v2[1] = v2[1] + rv * z;
        })
        if (!(ok = group_allsum<2>(v2, g, 5))) break;
        ++total_it;
        const float est = sqrtf(v2[0]);
        seg_end = est;
        if (!(est >= stop_abs)) break;  // reduced enough (or NaN)
        beta = v2[1] / guard_small(rz);
        rz = v2[1];
      }
      if (!ok) break;
      // Refinement: x += e in FP64; then r = Su - A x with the FP64
      // operator (needs every block's x: a barrier first).
      EAF_OWN_CELLS({ x[c] = x[c] + (double)e[c]; })
      if (!(ok = group_barrier(g))) break;
      double w64[1] = {0.0};
      EAF_OWN_CELLS({
        const double rv = b[c] - apply_row<SYM, double>(d, A64, x, c);
        s.r[c] = rv;
        w64[0] = w64[0] + rv * rv;
      })
      if (!(ok = group_allsum<1>(w64, g, 0))) break;
      ++outer;
      residual = sqrt(w64[0]) / bnorm;
      if (a.trace && g.bid == 0 && threadIdx.x == 0) {
        double* t = a.trace + 3 * (size_t)(outer - 1);
        t[0] = (double)(total_it - it_before);
        t[1] = seg_start > 0.f ? (double)seg_end / (double)seg_start : 0.0;
        t[2] = residual;
      }
    }
  }
#undef EAF_OWN_CELLS
  if (g.bid == 0 && threadIdx.x == 0) {
    SolveResult* res = a.ws.result;
    const int err = ld_volatile_i32(a.ws.err);
    res->status = err != 0 ? err : (isfinite(residual) ? EAF_OK : EAF_ENONFINITE);
    res->n_iter = total_it;
    res->n_outer = outer;
    res->sym = SYM ? 1 : 0;
    res->residual = residual;
    res->bnorm = bnorm;
  }
}

__global__ void __launch_bounds__(kMaxBlock) cg_mixed_kernel(MixArgs a) {
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
    mixed_body<true>(a, g);
  else
    mixed_body<false>(a, g);
}

struct BatchMixArgs {
  BatchTables t;
  int max_outer, max_inner;
  double tol, inner_tol;
  uint64_t timeout_ns;
};

__global__ void __launch_bounds__(kMaxBlock) batch_mixed_kernel(BatchMixArgs a) {
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
    MixArgs ma;
    ma.d = bs.d;
    ma.s = bs.s;
    ma.f = bs.f;
    ma.ws.part = g.part;
    ma.ws.counter = g.counter;
    ma.ws.err = a.t.err;
    ma.ws.result = bs.result;
    ma.max_outer = a.max_outer;
    ma.max_inner = a.max_inner;
    ma.tol = a.tol;
    ma.inner_tol = a.inner_tol;
    ma.timeout_ns = a.timeout_ns;
    ma.trace = nullptr;
    if (*bs.s.asym == 0)
      mixed_body<true>(ma, g);
    else
      mixed_body<false>(ma, g);
  }
}

}  // namespace

cudaError_t launch_batch_mixed(const BatchTables& t, int grid, int block,
                               int max_outer, int max_inner, double tol,
                               double inner_tol, uint64_t timeout_ns, cudaStream_t st) {
  BatchMixArgs a;
  a.t = t;
  a.max_outer = max_outer;
  a.max_inner = max_inner;
  a.tol = tol;
  a.inner_tol = inner_tol;
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
  return cudaLaunchKernelEx(&cfg, batch_mixed_kernel, a);
}

const void* batch_mixed_kernel_ptr() { return (const void*)batch_mixed_kernel; }

cudaError_t launch_cg_mixed(const MeshDims& d, const SysF64& s, const SysF32& f,
                            const GroupWs& ws, int max_outer, int max_inner,
                            double tol, double inner_tol, uint64_t timeout_ns,
                            int grid, int block, cudaStream_t st, double* trace) {
  MixArgs a;
  a.d = d;
  a.s = s;
  a.f = f;
  a.ws = ws;
  a.max_outer = max_outer;
  a.max_inner = max_inner;
  a.tol = tol;
  a.inner_tol = inner_tol;
  a.timeout_ns = timeout_ns;
  a.trace = trace;
  cudaError_t err = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (err == cudaSuccess) err = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (err != cudaSuccess) return err;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)cg_mixed_kernel, dim3(grid),
                                     dim3(block), args, 0, st);
}

const void* cg_mixed_kernel_ptr() { return (const void*)cg_mixed_kernel; }

}  // namespace eaf
