// Line-by-line TDMA sweeps and the transport residual on the device.
//
// tdma_3d_mpi (src/mod_solver_3d.f90:252-366, serial branch) solves, per
// sweep, every r line (loop k, then j), every theta line (k, then i) and
// every z line (j, then i) with the Thomas algorithm `tdma` (:22-46),
// refreshing the theta halos before each direction. Each line solve reads
// phi in place, so a line sees the NEW values of the lines solved before it
// (Gauss-Seidel between lines) and the OLD values of the lines after it. The
// kernel keeps exactly that: it is bit-identical to the sequential sweep.
//
// Schedule. In a direction the lines form a grid (a, b) -- a the inner loop
// index, b the outer -- and line (a, b) needs the new values of (a-1, b) and
// (a, b-1) only. One warp owns one index of the grid and solves its chain of
// lines in order: the in-chain dependency is the warp's own previous line,
// kept in shared memory; the cross-chain one is the neighbouring owner's
// line, which the owner also writes into a mailbox -- one slot per cell,
// marked empty with a signalling NaN that arithmetic never produces -- and
// the consumer polls the values themselves (bounded wait): one L2 round trip
// per hand-over and no fence, since the data is the signal. The consumer
// marks the slots empty again; slots alternate by sweep parity, and the
// grid barrier between directions orders a reset before the slot's next
// use. Owners are chosen so that the cross-chain value is the
// THIRD term of the reference's right-hand side
//   d = (Su + c1m*p1m) + c1p*p1p;  d = (d + c2m*p2m) + c2p*p2p
// (p1m the in-chain neighbour, p2m the cross-chain one): everything before
// it is summed while the warp waits. r lines: owner k, chain j; theta lines:
// owner k, chain i; z lines: owner i, chain j. The critical path is about
// (owners + chain) line solves plus one publish per owner.
//
// Lane 0 runs the Thomas recurrences (two correctly rounded divisions per
// cell, the reference's operation order); the other lanes gather and
// scatter the line. Built with -fmad=false like the CG unit.
#include <cuda_runtime.h>
#include <stdint.h>

#include "cg_common.cuh"
#include "cg_kernels.h"
#include "recipdiv.cuh"
#include "stencil.cuh"
#include "eafcg.h"

namespace eaf {
namespace {

struct TdmaArgs {
  HaloInputs in;  // aW..Su (phi unused: the kernel writes `phi`)
  double* phi;
  int nr, nth, nz;
  long long sx, sxy;  // halo strides of j and k
  int n_sweep;
  int lmax;
  double* mbox;       // hand-over slots, [2 parities][3 directions][n cells]
  double* fac;        // line factors, [3 directions][m, y, cp][n cells]
  GroupWs ws;
  uint64_t timeout_ns;
};

// One direction's geometry: chain index a (stride sa), owner index b
// (stride sb), line element e (stride se); cell (a, b, e) sits at halo
// index base + a*sa + b*sb + e*se. c1m/c1p the coefficients of the first
// neighbour pair of the right-hand side (stride s1; its minus side is the
// chain's previous line), c2m/c2p the second pair (stride s2; its minus
// side is the previous owner's line), lm/lp the in-line links.
struct Dir {
  int A, B, L;
  long long sa, sb, se, s1, s2;
  const double *c1m, *c1p, *c2m, *c2p, *lm, *lp;
};

__device__ __forceinline__ Dir make_dir(const TdmaArgs& a, int dir) {
  Dir d;
  const long long one = 1;
  if (dir == 0) {  // r lines: element i, chain j, owner k
    d.A = a.nth; d.B = a.nz; d.L = a.nr;
    d.sa = a.sx; d.sb = a.sxy; d.se = one;
    d.s1 = a.sx; d.c1m = a.in.aS; d.c1p = a.in.aN;
    d.s2 = a.sxy; d.c2m = a.in.aB; d.c2p = a.in.aT;
    d.lm = a.in.aW; d.lp = a.in.aE;
  } else if (dir == 1) {  // theta lines: element j, chain i, owner k
    d.A = a.nr; d.B = a.nz; d.L = a.nth;
    d.sa = one; d.sb = a.sxy; d.se = a.sx;
    d.s1 = one; d.c1m = a.in.aW; d.c1p = a.in.aE;
    d.s2 = a.sxy; d.c2m = a.in.aB; d.c2p = a.in.aT;
    d.lm = a.in.aS; d.lp = a.in.aN;
  } else {  // z lines: element k, chain j, owner i
    d.A = a.nth; d.B = a.nr; d.L = a.nz;
    d.sa = a.sx; d.sb = one; d.se = a.sxy;
    d.s1 = a.sx; d.c1m = a.in.aS; d.c1p = a.in.aN;
    d.s2 = one; d.c2m = a.in.aW; d.c2p = a.in.aE;
    d.lm = a.in.aB; d.lp = a.in.aT;
  }
  return d;
}

__device__ __forceinline__ double sign_small(double v) {
  return fabs(v) < kSmall ? copysign(kSmall, v) : v;
}

// Serial theta-periodic halo copy (src/mod_mpi_topology.f90:303-311) over
// all (i, k) columns of the halo layout, each column's four copies in the
// reference's statement order.
__device__ void theta_wrap(const TdmaArgs& a) {
  const long long ncol = (long long)(a.nr + 4) * (a.nz + 4);
  for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncol;
       col += (long long)gridDim.x * blockDim.x) {
    const long long i = col % (a.nr + 4), k = col / (a.nr + 4);
    double* p = a.phi + i + a.sxy * k;  // (i-1, j = -1, k-1) at p[0]
    auto J = [&](int j) { return (long long)(j + 1) * a.sx; };
    // With nth == 1 the second and fourth statements read the columns the
    // first and third just wrote; their values are taken from registers.
    const double v0 = __ldcg(p + J(a.nth));
    p[J(0)] = v0;
    p[J(-1)] = a.nth == 1 ? v0 : __ldcg(p + J(a.nth - 1));
    const double v1 = __ldcg(p + J(1));
    p[J(a.nth + 1)] = v1;
    p[J(a.nth + 2)] = a.nth == 1 ? v1 : __ldcg(p + J(2));
  }
}

constexpr int kTdmaMaxLine = 1024;  // 32 elements per lane in a hand-over mask

// Empty hand-over slot: a signalling NaN (IEEE arithmetic only delivers
// quiet NaNs, so no solution value has this pattern).
#define kEmptySlot __longlong_as_double(0x7ff000017ff00001ll)
constexpr unsigned long long kEmptyBits = 0x7ff000017ff00001ull;

// Line factors: the phi-independent half of `tdma` (src/mod_solver_3d.f90:
// 30-38) -- the guarded pivots m_i = b_i - a_i cp_{i-1} (b_1 for i = 1) and
// cp_i = c_i / m_i, in the reference's operations -- plus y_i = 1 / m_i, or
// 0 where m_i is outside the safe range of div_by_recip. One thread per line
// of every direction; the layout is [direction][m, y, cp][line][element].
__global__ void tdma_factor_kernel(TdmaArgs a) {
  const long long nA = (long long)a.nth * a.nz, nB = (long long)a.nr * a.nz,
                  nC = (long long)a.nr * a.nth;
  const long long n = (long long)a.nr * a.nth * a.nz;
  const long long base = 2 + 2 * a.sx + 2 * a.sxy;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nA + nB + nC;
       t += (long long)gridDim.x * blockDim.x) {
    int dir;
    long long line;
    if (t < nA) { dir = 0; line = t; }
    else if (t < nA + nB) { dir = 1; line = t - nA; }
    else { dir = 2; line = t - nA - nB; }
    const Dir d = make_dir(a, dir);
    const int ch = (int)(line % d.A), b = (int)(line / d.A);
    const long long q0 = base + ch * d.sa + b * d.sb;
    double* M = a.fac + (long long)dir * 3 * n + line * d.L;
    double* Y = M + n;
    double* CP = Y + n;
    double cp = 0.0;
    for (int e = 0; e < d.L; ++e) {
      const long long q = q0 + e * d.se;
      const double ai = -d.lm[q], bi = a.in.aP[q], ci = -d.lp[q];
      const double m = e == 0 ? sign_small(bi) : sign_small(bi - ai * cp);
      cp = ci / m;
      M[e] = m;
      Y[e] = exp_in_safe_range(m) ? 1.0 / m : 0.0;
      CP[e] = cp;
      const long long slot = (long long)dir * n + line * d.L + e;
      a.mbox[slot] = kEmptySlot;
      a.mbox[3 * n + slot] = kEmptySlot;
    }
  }
}

// ---------------------------------------------------------------------------
// Per owner, two warps: the LOADER fetches line ch+1 (coefficients, factors,
// the old neighbour values it needs, the end couplings) into one of two
// shared-memory buffers while the SOLVER finishes line ch; the solver then
// only forms the right-hand side from shared memory plus the two new values
// (its own previous line, the previous owner's mailbox) and runs the Thomas
// recurrences. Hand-shake: named barriers FULL_k / EMPTY_k per buffer k (a
// producer never arrives twice on one barrier before its consumer synced).
// ---------------------------------------------------------------------------
constexpr int kBarFull0 = 3, kBarEmpty0 = 5;  // FULL_k = 3 + k, EMPTY_k = 5 + k
constexpr int kTdmaBlock = 64;
constexpr int kBufArrays = 11;

struct LineBuf {
  double *su, *c1m, *c1t, *c2m, *c2t, *p1h, *p2h, *lo, *m, *y, *cp;
};

__device__ __forceinline__ LineBuf line_buf(double* base, int lmax) {
  LineBuf b;
  b.su = base;
  b.c1m = b.su + lmax;
  b.c1t = b.c1m + lmax;
  b.c2m = b.c1t + lmax;
  b.c2t = b.c2m + lmax;
  b.p1h = b.c2t + lmax;
  b.p2h = b.p1h + lmax;
  b.lo = b.p2h + lmax;
  b.m = b.lo + lmax;
  b.y = b.m + lmax;
  b.cp = b.y + lmax;
  return b;
}

// Loader: everything of line `ch` of owner `b` that does not depend on this
// sweep's new values. Products are formed as the reference forms them
// (c1p*p1p and c2p*p2p are added as whole terms); halo values for the
// first line of the chain (p1) and for owner 0 (p2).
__device__ __forceinline__ void load_line(const TdmaArgs& a, const Dir& d, const LineBuf& lb,
                                          double* ends, long long q0, int ch, int b,
                                          const double* fm, int lane) {
  const double* __restrict__ phi = a.phi;
  const double* __restrict__ Su = a.in.Su;
  const long long n = (long long)a.nr * a.nth * a.nz;
  for (int e = lane; e < d.L; e += 32) {
    const long long q = q0 + e * d.se;
    lb.su[e] = Su[q];
    lb.c1m[e] = d.c1m[q];
    lb.c1t[e] = d.c1p[q] * __ldcg(phi + q + d.s1);
    lb.c2m[e] = d.c2m[q];
    lb.c2t[e] = d.c2p[q] * __ldcg(phi + q + d.s2);
    if (ch == 0) lb.p1h[e] = __ldcg(phi + q - d.s1);
    if (b == 0) lb.p2h[e] = __ldcg(phi + q - d.s2);
    lb.lo[e] = -d.lm[q];
    lb.m[e] = __ldcg(fm + e);
    lb.y[e] = __ldcg(fm + n + e);
    lb.cp[e] = __ldcg(fm + 2 * n + e);
  }
  if (lane == 0) {
    const long long qL = q0 + (long long)(d.L - 1) * d.se;
    ends[0] = d.lm[q0] * __ldcg(phi + q0 - d.se);
    ends[1] = d.lp[qL] * __ldcg(phi + qL + d.se);
  }
}

// The phi-dependent half of tdma (src/mod_solver_3d.f90:32-45), lane 0:
// dp_1 = d_1 / m_1, dp_i = (d_i - a_i dp_{i-1}) / m_i, x_i = dp_i - cp_i x_{i+1}.
// The forward pass runs on the correction path only, its range conditions
// OR-ed off the dependent chain; a line with any operand outside the safe
// range (rare) is redone with `/` throughout. A zero numerator is exact on
// this path as q = t*y itself (the correction would turn -0 into +0).
__device__ __forceinline__ void thomas_line(const LineBuf& lb, const double* __restrict__ rhs,
                                            double* __restrict__ dpa,
                                            double* __restrict__ x, int L) {
  const double* __restrict__ lo = lb.lo;
  const double* __restrict__ mm = lb.m;
  const double* __restrict__ yy = lb.y;
  const double* __restrict__ cpa = lb.cp;
  bool ok = yy[0] != 0.0 && (rhs[0] == 0.0 || exp_in_safe_range(rhs[0]));
  double dp;
  {
    const double t = rhs[0], q = t * yy[0];
    const double c = __fma_rn(__fma_rn(-q, mm[0], t), yy[0], q);
    dp = t == 0.0 ? q : c;
  }
  dpa[0] = dp;
  for (int i = 1; i < L; ++i) {
    const double y = yy[i], m = mm[i];
    const double t = rhs[i] - lo[i] * dp;
    ok = ok & (y != 0.0) & (t == 0.0 || exp_in_safe_range(t));
    const double q = t * y;
    const double c = __fma_rn(__fma_rn(-q, m, t), y, q);
    dp = t == 0.0 ? q : c;
    dpa[i] = dp;
  }
  if (!ok) {
    dp = rhs[0] / mm[0];
    dpa[0] = dp;
    for (int i = 1; i < L; ++i) {
      dp = (rhs[i] - lo[i] * dp) / mm[i];
      dpa[i] = dp;
    }
  }
  double xv = dp;
  x[L - 1] = xv;
  for (int i = L - 2; i >= 0; --i) {
    xv = dpa[i] - cpa[i] * xv;
    x[i] = xv;
  }
}

// Polls the previous owner's mailbox for line values (bounded); completes
// rhs_e = (rhs_e + c2m_e * p2m_e) + c2t_e as they arrive and empties the
// slots. False if the wait gave up.
__device__ bool take_mailbox(const TdmaArgs& a, unsigned long long* slot, const LineBuf& lb,
                             double* rhs, int L, int lane) {
  unsigned pend = 0;
  for (int k = 0; lane + 32 * k < L; ++k) pend |= 1u << k;
  uint64_t t0 = 0;
  uint32_t spins = 0;
  for (;;) {
    for (int k = 0; lane + 32 * k < L; ++k) {
      if (!(pend & (1u << k))) continue;
      const int e = lane + 32 * k;
      const unsigned long long v = ld_relaxed_u64(slot + e);
      if (v == kEmptyBits) continue;
      const double t = rhs[e] + lb.c2m[e] * __longlong_as_double((long long)v);
      rhs[e] = t + lb.c2t[e];
      slot[e] = kEmptyBits;
      pend &= ~(1u << k);
    }
    if (!__any_sync(0xffffffffu, pend != 0)) return true;
    if ((++spins & 63u) == 0) {
      int stop = 0;
      if (lane == 0) {
        if (spins == 64u) t0 = global_ns();
        if (ld_volatile_i32(a.ws.err) != 0) {
          stop = 1;
        } else if (global_ns() - t0 > a.timeout_ns) {
          atomicCAS(a.ws.err, 0, (int)EAF_ETIMEOUT);
          stop = 1;
        }
      }
      if (__shfl_sync(0xffffffffu, stop, 0)) return false;
    }
  }
}

__global__ void __launch_bounds__(kTdmaBlock) tdma_kernel(TdmaArgs a) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double s_ends[2][2];
  const LineBuf buf0 = line_buf(sm, a.lmax);
  const LineBuf buf1 = line_buf(sm + kBufArrays * a.lmax, a.lmax);
  double* s_x = sm + 2 * kBufArrays * a.lmax;
  double* s_rhs = s_x + a.lmax;
  double* s_dp = s_rhs + a.lmax;
  const int lane = threadIdx.x & 31;
  const bool loader = threadIdx.x >= 32;
  Group g;
  g.counter = a.ws.counter;
  g.err = a.ws.err;
  g.part = a.ws.part;
  g.stage = nullptr;
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.timeout_ns = a.timeout_ns;
  g.epoch = 0;
  const long long base = 2 + 2 * a.sx + 2 * a.sxy;  // cell (1, 1, 1)
  double* __restrict__ phi = a.phi;
  bool ok = true;
  for (int sweep = 1; sweep <= a.n_sweep && ok; ++sweep) {
    for (int dir = 0; dir < 3 && ok; ++dir) {
      if (!(ok = group_barrier<1>(g))) break;
      theta_wrap(a);
      if (!(ok = group_barrier<1>(g))) break;
      const Dir d = make_dir(a, dir);
      const long long ncell = (long long)a.nr * a.nth * a.nz;
      const double* fdir = a.fac + (long long)dir * 3 * ncell;
      double* mb = a.mbox + ((long long)(sweep & 1) * 3 + dir) * ncell;
      for (int b = blockIdx.x; b < d.B; b += gridDim.x) {
        const long long qb = base + b * d.sb;
        const long long lines_b = (long long)b * d.A * d.L;  // line (0, b)
        if (loader) {
          for (int ch = 0; ch < d.A; ++ch) {
            const int k = ch & 1;
            if (ch >= 2) named_sync(kBarEmpty0 + k, kTdmaBlock);
            load_line(a, d, k ? buf1 : buf0, s_ends[k], qb + ch * d.sa, ch, b,
                      fdir + lines_b + (long long)ch * d.L, lane);
            named_arrive(kBarFull0 + k, kTdmaBlock);
          }
          continue;
        }
        double* mine = mb + lines_b;
        unsigned long long* from =
            b > 0 ? reinterpret_cast<unsigned long long*>(mb + lines_b - (long long)d.A * d.L)
                  : nullptr;
        const bool feeds = b + 1 < d.B;
        bool live = true;  // false after a wait gave up: keep the hand-shake only
        for (int ch = 0; ch < d.A; ++ch) {
          const int k = ch & 1;
          const LineBuf lb = k ? buf1 : buf0;
          named_sync(kBarFull0 + k, kTdmaBlock);
          if (live) {
            const long long q0 = qb + ch * d.sa;
            for (int e = lane; e < d.L; e += 32) {
              const double p1m = ch == 0 ? lb.p1h[e] : s_x[e];
              double t = lb.su[e] + lb.c1m[e] * p1m;
              t = t + lb.c1t[e];
              if (b == 0) {
                t = t + lb.c2m[e] * lb.p2h[e];
                t = t + lb.c2t[e];
              }
              s_rhs[e] = t;
            }
            if (b > 0 && !take_mailbox(a, from + (long long)ch * d.L, lb, s_rhs, d.L, lane))
              live = false;
            __syncwarp();
            if (live) {
              if (lane == 0) {
                // lagged couplings of the segment ends (:299-302, :325-328, :352-355)
                s_rhs[0] = s_rhs[0] + s_ends[k][0];
                s_rhs[d.L - 1] = s_rhs[d.L - 1] + s_ends[k][1];
                thomas_line(lb, s_rhs, s_dp, s_x, d.L);
              }
              __syncwarp();
              for (int e = lane; e < d.L; e += 32) {
                const double xv = s_x[e];
                if (feeds) mine[(long long)ch * d.L + e] = xv;
                phi[q0 + e * d.se] = xv;
              }
              __syncwarp();
            }
          }
          if (ch + 2 < d.A) named_arrive(kBarEmpty0 + k, kTdmaBlock);
        }
      }
      // A solver whose wait gave up kept the hand-shake and set the error
      // word; the other waits see it and give up too, so every warp reaches
      // the next group barrier and the launch ends with EAF_ETIMEOUT.
    }
  }
}

// ---------------------------------------------------------------------------
// compute_residual_3d_mpi (src/mod_solver_3d.f90:625-694), serial: one pass
// over the interior in the blocks' contiguous slices, the two sums reduced
// with the deterministic group all-reduce (the CG dots' association).
// ---------------------------------------------------------------------------
struct ResArgs {
  HaloInputs in;
  const double* phi;
  MeshDims d;
  long long sx, sxy;
  GroupWs ws;
  uint64_t timeout_ns;
};

__global__ void __launch_bounds__(1024) residual_kernel(ResArgs a) {
  Group g;
  g.counter = a.ws.counter;
  g.err = a.ws.err;
  g.part = a.ws.part;
  g.stage = group_stage_smem();
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.timeout_ns = a.timeout_ns;
  g.epoch = 0;
  const Slice own = own_slice(a.d.n, g.nb, g.bid);
  double v[2] = {0.0, 0.0};
  const HaloInputs& in = a.in;
  for (int c = own.begin + (int)threadIdx.x; c < own.end; c += blockDim.x) {
    int i, j, k;
    cell_ijk(a.d, c, i, j, k);
    const long long q = (i + 2) + a.sx * (j + 2) + a.sxy * (k + 2);
    const double P = in.aP[q], W = in.aW[q], E = in.aE[q], S = in.aS[q], N = in.aN[q],
                 B = in.aB[q], T = in.aT[q], U = in.Su[q];
    if (P == 1.0 && W == 0.0 && E == 0.0 && S == 0.0 && N == 0.0 && B == 0.0 &&
        T == 0.0) {
      v[0] = v[0] + 0.0;
      v[1] = v[1] + 0.0;
      continue;
    }
    const double* ph = a.phi;
    const double pc = ph[q];
    double r = U - P * pc + S * ph[q - a.sx] + N * ph[q + a.sx];
    r = r + W * ph[q - 1] + E * ph[q + 1];
    r = r + B * ph[q - a.sxy] + T * ph[q + a.sxy];
    const double t = fabs(U) + fabs(P * pc) + kSmall;
    v[0] = v[0] + r * r;
    v[1] = v[1] + t * t;
  }
  const bool ok = group_allsum<2>(v, g, 0);
  if (g.bid == 0 && threadIdx.x == 0) {
    SolveResult* res = a.ws.result;
    const int err = ld_volatile_i32(a.ws.err);
    res->status = err != 0 ? err : (ok ? EAF_OK : EAF_ETIMEOUT);
    res->n_iter = 0;
    res->n_outer = 0;
    res->sym = 0;
    res->residual = sqrt(v[0]) / (sqrt(v[1]) + kSmall);
    res->bnorm = 0.0;
  }
}

// Diagnostic: div_by_recip against `/`, bit for bit, on generated pairs.
// Case mix per index: random sign, mantissa and exponent in [-540, 540]
// (both paths); t = m * k for small integers k (exact quotients); t one ulp
// off m * k (quotients next to halfway points); zeros, infinities, NaN.
__device__ __forceinline__ unsigned long long splitmix(unsigned long long x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

__device__ double gen_double(unsigned long long r, int emin, int emax) {
  const unsigned long long mant = r & 0xfffffffffffffull;
  const int span = emax - emin + 1;
  const int ex = emin + (int)((r >> 52) % (unsigned long long)span);
  const unsigned long long sign = (r >> 63) << 63;
  return __longlong_as_double((long long)(sign | ((unsigned long long)(ex + 1023) << 52) | mant));
}

__global__ void div_check_kernel(long long n, unsigned long long seed,
                                 unsigned long long* counts) {
  unsigned long long bad = 0, fast = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long r1 = splitmix(seed ^ (2 * (unsigned long long)i));
    const unsigned long long r2 = splitmix(seed ^ (2 * (unsigned long long)i + 1));
    double t, m;
    switch ((int)(i & 7)) {
      case 0: case 1: case 2:
        t = gen_double(r1, -540, 540);
        m = gen_double(r2, -540, 540);
        break;
      case 3: case 4: {
        m = gen_double(r2, -400, 400);
        const double k = (double)((long long)(r1 % 2000001ull) - 1000000);
        t = m * k;
        break;
      }
      case 5: case 6: {
        m = gen_double(r2, -400, 400);
        const double k = (double)((long long)(r1 % 2001ull) - 1000) + 0.5;
        const double p = m * k;
        t = (r1 >> 40) & 1 ? nextafter(p, 1e308) : nextafter(p, -1e308);
        break;
      }
      default: {
        const double specials[6] = {0.0, -0.0, __longlong_as_double(0x7ff0000000000000ll),
                                    __longlong_as_double((long long)0xfff0000000000000ull),
                                    __longlong_as_double(0x7ff8000000000000ll), 1e-310};
        t = (r1 & 1) ? specials[(r1 >> 1) % 6] : gen_double(r1, -540, 540);
        m = (r2 & 1) ? specials[(r2 >> 1) % 6] : gen_double(r2, -540, 540);
        break;
      }
    }
    const bool m_ok = exp_in_safe_range(m);
    const double y = m_ok ? 1.0 / m : 0.0;
    const double a = div_by_recip(t, m, y, m_ok);
    const double b = t / m;
    const bool same = (__double_as_longlong(a) == __double_as_longlong(b)) ||
                      (a != a && b != b);
    bad += same ? 0 : 1;
    fast += (m_ok && (t == 0.0 || exp_in_safe_range(t))) ? 1 : 0;
  }
  atomicAdd(counts, bad);
  atomicAdd(counts + 1, fast);
}

}  // namespace

size_t tdma_mailbox_doubles(int nr, int nth, int nz) {
  return (size_t)6 * nr * nth * nz;
}

int tdma_grid(int nr, int nth, int nz) {
  // Owners per direction: k (r lines), k (theta lines), i (z lines).
  return nz > nr ? nz : nr;
}

size_t tdma_factor_doubles(int nr, int nth, int nz) {
  return (size_t)9 * nr * nth * nz;
}

cudaError_t launch_tdma_f64(const HaloInputs& in, double* phi, int nr, int nth, int nz,
                            int n_sweep, double* mbox, double* fac, const GroupWs& ws,
                            uint64_t timeout_ns, cudaStream_t st) {
  if (nr > kTdmaMaxLine || nth > kTdmaMaxLine || nz > kTdmaMaxLine)
    return cudaErrorInvalidValue;
  TdmaArgs a;
  a.in = in;
  a.phi = phi;
  a.nr = nr;
  a.nth = nth;
  a.nz = nz;
  a.sx = nr + 4;
  a.sxy = (long long)(nr + 4) * (nth + 4);
  a.n_sweep = n_sweep;
  int lmax = nr > nth ? nr : nth;
  if (nz > lmax) lmax = nz;
  a.lmax = lmax;
  a.mbox = mbox;
  a.fac = fac;
  a.ws = ws;
  a.timeout_ns = timeout_ns;
  const int grid = tdma_grid(nr, nth, nz);
  const size_t smem = (size_t)(2 * kBufArrays + 3) * lmax * sizeof(double);
  std::lock_guard<std::mutex> attr_lock(launch_attr_mutex());
  cudaError_t e = cudaSuccess;
  if (smem > 48 * 1024)
    e = cudaFuncSetAttribute((const void*)tdma_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    const long long lines = (long long)nth * nz + (long long)nr * nz + (long long)nr * nth;
    const int fb = 128;
    long long fg = (lines + fb - 1) / fb;
    if (fg > 4096) fg = 4096;
    tdma_factor_kernel<<<(unsigned)fg, fb, 0, st>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)tdma_kernel, dim3(grid), dim3(kTdmaBlock), args,
                                     smem, st);
}

cudaError_t launch_residual_f64(const HaloInputs& in, const double* phi, const MeshDims& d,
                                const GroupWs& ws, uint64_t timeout_ns, int grid, int block,
                                cudaStream_t st) {
  ResArgs a;
  a.in = in;
  a.phi = phi;
  a.d = d;
  a.sx = d.nr + 4;
  a.sxy = (long long)(d.nr + 4) * (d.nth + 4);
  a.ws = ws;
  a.timeout_ns = timeout_ns;
  cudaError_t e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)residual_kernel, dim3(grid), dim3(block),
                                     args, 0, st);
}

const void* tdma_kernel_ptr() { return (const void*)tdma_kernel; }
const void* residual_kernel_ptr() { return (const void*)residual_kernel; }

cudaError_t run_div_check(long long n, unsigned long long seed, unsigned long long* counts,
                          cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  div_check_kernel<<<592, 256, 0, st>>>(n, seed, counts);
  return cudaGetLastError();
}

}  // namespace eaf
