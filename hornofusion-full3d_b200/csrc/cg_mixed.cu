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
// Refinement policy: an inner segment runs FP32 CG on A e = r. When its
// estimated residual has dropped by `inner_tol` since the segment began
// (or suggests the outer tolerance is met, or the segment reached
// max_inner iterations), the correction is folded into x in FP64, the true
// residual is recomputed in FP64 and replaces the FP32 estimate. The search
// direction is kept across the replacement (the "reliable update" scheme of
// Sleijpen & van der Vorst, Computing 56 (1996) 141-163), so the Krylov
// progress of the FP32 iterations is not thrown away at every refinement.
#include <math.h>

#include "cg_kernels.h"
#include "stencil.cuh"

namespace eaf {
namespace {

constexpr int kUnroll = 4;
constexpr int kMaxBlock = 1024;

struct MixArgs {
  MeshDims d;
  SysF64 s;
  SysF32 f;
  GroupWs ws;
  int max_outer, max_inner;
  double tol, inner_tol;
  uint64_t timeout_ns;
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
  float* __restrict__ p = f.p;
  float* __restrict__ q = f.q;
  float* __restrict__ e = f.e;
#define EAF_OWN_CELLS(...) EAF_FOR_OWN(own, kUnroll, c, __VA_ARGS__)

  // Setup: FP32 coefficient copies, rs = r, e = 0, z = rs/d, p = z.
  double v64[2] = {0.0, 0.0};  // ||Su||^2, ||r||^2 (FP64)
  float v32[2] = {0.f, 0.f};   // rs.rs, rs.z     (FP32)
  EAF_OWN_CELLS({
    const float dv = (float)s.aP[c];
    f.aP[c] = dv;
    f.aE[c] = (float)s.aE[c];
    f.aN[c] = (float)s.aN[c];
    f.aT[c] = (float)s.aT[c];
    if (!SYM) {
      f.aW[c] = (float)s.aW[c];
      f.aS[c] = (float)s.aS[c];
      f.aB[c] = (float)s.aB[c];
    }
    const double bv = b[c], rv = s.r[c];
    const float r32 = (float)rv;
    const float z = r32 / guard_small(fabsf(dv));
    rs[c] = r32;
    p[c] = z;
    e[c] = 0.f;
    v64[0] = v64[0] + bv * bv;
    v64[1] = v64[1] + rv * rv;
    v32[0] = v32[0] + r32 * r32;
    v32[1] = v32[1] + r32 * z;
  })
  bool ok = group_allsum<2>(v64, g, 0);
  ok = ok && group_allsum<2>(v32, g, 2);
  const double bnorm = sqrt(v64[0]);
  double residual = 0.0;
  int total_it = 0, outer = 0;
  if (ok && !(bnorm < kSmall)) {
    residual = sqrt(v64[1]) / bnorm;
    float rz = v32[1];
    float seg_start = sqrtf(v32[0]);
    const float target_abs = (float)(a.tol * bnorm);
    int seg_it = 0;
    bool done = !(residual >= a.tol) || a.max_outer < 1;  // converged or NaN
    while (!done) {
      // S0: q = A p (FP32), p.q
      float v1[1] = {0.f};
      EAF_OWN_CELLS({
        const float qv = apply_row<SYM, float>(d, A32, p, c);
        q[c] = qv;
        v1[0] = v1[0] + p[c] * qv;
      })
      if (!(ok = group_allsum<1>(v1, g, 4))) break;
      const float pq = v1[0];
      const bool breakdown = !(fabsf(pq) >= 1.0e-30f);
      const float alpha = breakdown ? 0.f : rz / pq;
      // S1: e += alpha p; rs -= alpha q; rs.rs and rs.z
      float v2[2] = {0.f, 0.f};
      EAF_OWN_CELLS({
        const float pv = p[c], qv = q[c];
        e[c] = e[c] + alpha * pv;
        const float rv = rs[c] - alpha * qv;
        rs[c] = rv;
        const float z = rv / guard_small(fabsf(dP[c]));
        v2[0] = v2[0] + rv * rv;
        v2[1] = v2[1] + rv * z;
      })
      if (!(ok = group_allsum<2>(v2, g, 5))) break;
      if (!breakdown) {
        ++total_it;
        ++seg_it;
      }
      float rz_new = v2[1];
      const float est = sqrtf(v2[0]);
      if (breakdown || est < (float)a.inner_tol * seg_start || est < target_abs ||
          seg_it >= a.max_inner || !(est == est)) {
        // Refinement: x += e (FP64), then r = Su - A x in FP64 replaces rs.
        EAF_OWN_CELLS({
          x[c] = x[c] + (double)e[c];
          e[c] = 0.f;
        })
        if (!(ok = group_barrier(g))) break;
        double w64[1] = {0.0};
        float w32[2] = {0.f, 0.f};
        EAF_OWN_CELLS({
          const double rv = b[c] - apply_row<SYM, double>(d, A64, x, c);
          const float r32 = (float)rv;
          rs[c] = r32;
          const float z = r32 / guard_small(fabsf(dP[c]));
          w64[0] = w64[0] + rv * rv;
          w32[0] = w32[0] + r32 * r32;
          w32[1] = w32[1] + r32 * z;
        })
        if (!(ok = group_allsum<1>(w64, g, 0))) break;
        if (!(ok = group_allsum<2>(w32, g, 2))) break;
        ++outer;
        residual = sqrt(w64[0]) / bnorm;
        if (!(residual >= a.tol) || outer >= a.max_outer || breakdown) break;
        rz_new = w32[1];
        seg_start = sqrtf(w32[0]);
        seg_it = 0;
      }
      const float beta = rz_new / guard_small(rz);
      rz = rz_new;
      // S2: p = z + beta p
      EAF_OWN_CELLS({
        const float z = rs[c] / guard_small(fabsf(dP[c]));
        p[c] = z + beta * p[c];
      })
      if (!(ok = group_barrier(g))) break;
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

}  // namespace

cudaError_t launch_cg_mixed(const MeshDims& d, const SysF64& s, const SysF32& f,
                            const GroupWs& ws, int max_outer, int max_inner,
                            double tol, double inner_tol, uint64_t timeout_ns,
                            int grid, int block, cudaStream_t st) {
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
  cudaError_t err = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (err == cudaSuccess) err = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (err != cudaSuccess) return err;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)cg_mixed_kernel, dim3(grid),
                                     dim3(block), args, 0, st);
}

const void* cg_mixed_kernel_ptr() { return (const void*)cg_mixed_kernel; }

}  // namespace eaf
