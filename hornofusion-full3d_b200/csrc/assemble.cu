// Assembly of the pressure-correction equation on the device: the serial
// code of solve_pressure_correction before the CG (src/mod_pressure_3d.f90:
// 135-310). Four launches:
//   G. cell gradients (cell_gradients :621-651) of the liquid and, for the
//      gas, the vertical one with the liquid weight (gas_gz :421-440; its r
//      and theta gradients equal the liquid's); one thread per halo element,
//      theta halo rows computing their source row of the periodic copy, so
//      neither a clearing pass nor a halo pass is needed;
//   F. faces: add_phase_contribution (:469-619) evaluates every interior
//      face twice, once from each side, and both evaluations are the same
//      arithmetic (the two-term sums commute exactly); so each face is
//      computed once, by the cell on its + side (its W, S and B faces), per
//      phase: link and open flags, and for r and z faces the coefficient
//      and the flux, for theta faces af * d_f and af * u_f (the reference
//      multiplies those by the area of the cell that is adding the face,
//      which differs between the two sides);
//   C. cells: one thread per halo element: every output zeroed; in interior
//      cells the six faces of each phase added in the reference's order, the
//      compressibility source (:228-247), trivial rows and the diagonal
//      (:250-285) and the boundary folding (apply_pressure_bc,
//      src/mod_boundary_3d.f90:180-277); per-block partials of flux_ref and
//      sum |Su|;
//   R. the block partials folded in a fixed order into the residual.
// Built with -fmad=false, like the other units that must match the
// reference's non-FMA arithmetic.
#include <cuda_runtime.h>
#include <stdint.h>

#include "cg_common.cuh"
#include "cg_kernels.h"
#include "recipdiv.cuh"
#include "eafcg.h"

namespace eaf {
namespace {

constexpr double kS = 1.0e-30;          // SMALL
constexpr double kGrav = 9.81;          // GRAVITY, src/mod_constants.f90:18
constexpr double kCompliance = 1.0e-6;  // PP_COMPLIANCE, src/mod_pressure_3d.f90:50
constexpr double kCompCap = 0.2;        // COMP_SRC_CAP, :56
constexpr double kP0 = 101325.0;        // P0_THERMO, :68
constexpr double kCsound = 4000.0;      // C_SOUND_LIQ, :72
constexpr double kTminGas = 100.0;      // T_MIN_GAS, src/mod_constants.f90:148
constexpr double kRoomEps = 1.0e-4;     // ROOM_EPS, src/mod_pressure_3d.f90:662
constexpr int kAsmBlock = 256;

// Face values of one phase, per halo element (its W, S and B faces).
struct FacePhase {
  double *cW, *fW;  // r face: coefficient, flux
  double *dS, *uS;  // theta face: af * d_f, af * u_f
  double *cB, *fB;  // z face: coefficient, flux
};
// Open-face bits per element: liquid W, S, B = 1, 2, 4; gas = 8, 16, 32.
constexpr unsigned kBitW = 1, kBitS = 2, kBitB = 4, kGasShift = 3;

struct AsmArgs {
  eaf_assembly_fields_t f;
  double *gr, *gth, *gz_l, *gz_g;  // gradient scratch (halo layout)
  FacePhase fl, fg;                // face scratch, liquid and gas
  unsigned char* open;             // open-face bits
  double* part;                    // [2][grid] block partials
  double* result;                  // residual
  int nr, nth, nz;
  unsigned sx, sxy, rows, nh;      // halo strides, theta rows, elements
};

template <typename T>
__device__ __forceinline__ T ld(const T* p, unsigned q) {
  return __ldg(p + q);
}

// Cell indices of the 7-point stencil around q: c, w, e, s, n, b, t.
struct Stencil {
  unsigned q[7];
  __device__ Stencil(unsigned c, unsigned sx, unsigned sxy)
      : q{c, c - 1, c + 1, c - sx, c + sx, c - sxy, c + sxy} {}
};
enum { C = 0, W = 1, E = 2, S = 3, N = 4, B = 5, T = 6 };

// pgrad (src/mod_constants.f90:274-287)
__device__ __forceinline__ double pgrad(double pm, double p0, double pp, double xm, double x0,
                                        double xp, bool okm, bool okp) {
  if (okm && okp) return (pp - pm) / (xp - xm);
  if (okp) return (pp - p0) / (xp - x0);
  if (okm) return (p0 - pm) / (x0 - xm);
  return 0.0;
}

// liq_weight_f (:407-417) from the liquid's mask, fraction, density and
// temperature of the lower cell (a) and the upper one (b).
__device__ __forceinline__ double liq_weight(double beta, double ta, bool la, double aa,
                                             double ra, double Ta, bool lb, double ab,
                                             double rb, double Tb) {
  return 0.5 * kGrav *
         ((la ? 1.0 : 0.0) * aa * ra * (1.0 - beta * (Ta - ta)) +
          (lb ? 1.0 : 0.0) * ab * rb * (1.0 - beta * (Tb - ta)));
}

// Halo element q -> (i, j, k), 1-based interior indices.
__device__ __forceinline__ void cell_of(const AsmArgs& a, unsigned q, int& i, int& j, int& k) {
  const unsigned u = q / a.sx;
  i = (int)(q - u * a.sx) - 1;
  const unsigned v = u / a.rows;
  j = (int)(u - v * a.rows) - 1;
  k = (int)v - 1;
}

// Every load of a cell is issued before the first decision that depends on
// one: the stencil's masks and pressures, the coordinates, and (gas) the
// liquid columns for the weights.
template <bool GAS_IN>
__global__ void __launch_bounds__(kAsmBlock, 4) asm_gradient_kernel(AsmArgs a) {
  const eaf_assembly_fields_t& f = a.f;
  for (unsigned qd = blockIdx.x * blockDim.x + threadIdx.x; qd < a.nh;
       qd += gridDim.x * blockDim.x) {
    int i, jd, k;
    cell_of(a, qd, i, jd, k);
    double gr = 0.0, gth = 0.0, gzl = 0.0, gzg = 0.0;
    if (i >= 1 && i <= a.nr && k >= 1 && k <= a.nz) {
      // source row of the periodic copy (src/mod_mpi_topology.f90:303-311),
      // including the nth == 1 case where the second and fourth copies read
      // rows the first and third wrote
      int j = jd;
      if (jd == 0) j = a.nth;
      else if (jd == -1) j = a.nth == 1 ? 1 : a.nth - 1;
      else if (jd == a.nth + 1) j = 1;
      else if (jd == a.nth + 2) j = a.nth == 1 ? 1 : 2;
      const Stencil st(qd + a.sx * (unsigned)(j - jd), a.sx, a.sxy);
      int ct[7], al[7], ag[7];
      double p[7];
#pragma unroll
      for (int m = 0; m < 7; ++m) {
        ct[m] = ld(f.cell_type, st.q[m]);
        al[m] = ld(f.act_l, st.q[m]);
        ag[m] = ld(f.act_g, st.q[m]);
        p[m] = ld(f.p, st.q[m]);
      }
      const double r0 = ld(f.r, i), r1 = ld(f.r, i + 1), r2 = ld(f.r, i + 2);
      const double t0 = ld(f.theta, j), t1 = ld(f.theta, j + 1), t2 = ld(f.theta, j + 2);
      const double z0 = ld(f.z, k), z1 = ld(f.z, k + 1), z2 = ld(f.z, k + 2);
      double la[3], lr[3], lT[3];  // liquid at c, b, t
      if (GAS_IN) {
        const int cbt[3] = {C, B, T};
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          la[m] = ld(f.liq.alpha, st.q[cbt[m]]);
          lr[m] = ld(f.liq.rho, st.q[cbt[m]]);
          lT[m] = ld(f.liq_T, st.q[cbt[m]]);
        }
      }
      bool pv[7];
#pragma unroll
      for (int m = 0; m < 7; ++m) pv[m] = (ct[m] != 0) & ((al[m] != 0) | (ag[m] != 0));
      if (ct[C] != 0) {
        gr = pgrad(p[W], p[C], p[E], r0, r1, r2, i > 1 && pv[W], i < a.nr && pv[E]);
        gth = pgrad(p[S], p[C], p[N], r1 * t0, r1 * t1, r1 * t2, pv[S], pv[N]);
        const bool okm = k > 1 && pv[B], okp = k < a.nz && pv[T];
        gzl = pgrad(p[B], p[C], p[T], z0, z1, z2, okm, okp);
        if (GAS_IN) {
          const double beta = f.beta_expansion, ta = f.T_ambient;
          double gb = 0.0, gt = 0.0;
          if (okm)
            gb = (p[C] - p[B]) / (z1 - z0) +
                 liq_weight(beta, ta, al[B] != 0, la[1], lr[1], lT[1], al[C] != 0, la[0],
                            lr[0], lT[0]);
          if (okp)
            gt = (p[T] - p[C]) / (z2 - z1) +
                 liq_weight(beta, ta, al[C] != 0, la[0], lr[0], lT[0], al[T] != 0, la[2],
                            lr[2], lT[2]);
          if (okm && okp) gzg = 0.5 * (gb + gt);
          else if (okp) gzg = gt;
          else if (okm) gzg = gb;
        }
      }
    }
    a.gr[qd] = gr;
    a.gth[qd] = gth;
    a.gz_l[qd] = gzl;
    if (GAS_IN) a.gz_g[qd] = gzg;
  }
}

// face_open (:660-668)
template <bool ISG, bool ROOM>
__device__ __forceinline__ bool face_open(double u_f, double room_neg, double room_pos) {
  if (ISG || !ROOM) return true;
  bool open = true;
  if (u_f > 0.0 && room_pos <= kRoomEps) open = false;
  if (u_f < 0.0 && room_neg <= kRoomEps) open = false;
  return open;
}

// Lower faces W, S, B of element q (index f = 0, 1, 2; lower neighbour x),
// shared by both phases: the distance between the cell centres and its
// reciprocal, the pressure term dp / delta of u_f, the area (r and z).
struct LowerFaces {
  unsigned q, x[3];
  int ct[4];  // q, w, s, b
  double p[4], vol[4], room[4];
  double delta[3], y[3], gp[3], area[3];
  bool ok[3];
};

// The three lower faces of one phase (add_phase_contribution, each face as
// the reference evaluates it from either side): writes the face values and
// returns the open bits W, S, B.
template <bool ISG, bool ROOM>
__device__ __forceinline__ unsigned phase_faces(const AsmArgs& a, const LowerFaces& L,
                                                const eaf_phase_state_t& ph, const int* act,
                                                const double* gz, double lw_b,
                                                const FacePhase& out) {
  const unsigned q = L.q;
  const int ac_q = ld(act, q);
  const double al_q = ld(ph.alpha, q);
  const double* apd[3] = {ph.aP_ur, ph.aP_uth, ph.aP_uz};
  const double* ud[3] = {ph.ur, ph.uth, ph.uz};
  const double* gd[3] = {a.gr, a.gth, gz};
  int ac_x[3];
  double al_x[3], ap_q[3], ap_x[3], u_q[3], u_x[3], g_q[3], g_x[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const unsigned x = L.x[f];
    ac_x[f] = ld(act, x);
    al_x[f] = ld(ph.alpha, x);
    ap_q[f] = ld(apd[f], q);
    ap_x[f] = ld(apd[f], x);
    u_q[f] = ld(ud[f], q);
    u_x[f] = ld(ud[f], x);
    g_q[f] = ld(gd[f], q);
    g_x[f] = ld(gd[f], x);
  }
  const double lw[3] = {0.0, 0.0, lw_b};
  unsigned bits = 0;
  double af[3], d_f[3], u_f[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    d_f[f] = 0.5 * (al_q * L.vol[0] / fmax(ap_q[f], kS) +
                    al_x[f] * L.vol[f + 1] / fmax(ap_x[f], kS));
    af[f] = 0.5 * (al_q + al_x[f]);
    u_f[f] = 0.5 * (u_q[f] + u_x[f]) + d_f[f] * (0.5 * (g_q[f] + g_x[f]) - L.gp[f] - lw[f]);
    const bool link = (L.ct[0] != 0) & (ac_q != 0) & (L.ct[f + 1] != 0) & (ac_x[f] != 0);
    if (link && face_open<ISG, ROOM>(u_f[f], L.room[f + 1], L.room[0])) bits |= 1u << f;
  }
  out.cW[q] = div_by_recip(af[0] * d_f[0] * L.area[0], L.delta[0], L.y[0], L.ok[0]);
  out.fW[q] = af[0] * u_f[0] * L.area[0];
  out.dS[q] = af[1] * d_f[1];
  out.uS[q] = af[1] * u_f[1];
  out.cB[q] = div_by_recip(af[2] * d_f[2] * L.area[2], L.delta[2], L.y[2], L.ok[2]);
  out.fB[q] = af[2] * u_f[2] * L.area[2];
  return bits;
}

// One thread per halo element whose lower faces some interior cell adds:
// i in 1..nr+1, j in 1..nth+1, k in 1..nz+1 (the others are never read).
template <bool GAS_IN, bool ROOM>
__global__ void __launch_bounds__(kAsmBlock, 2) asm_face_kernel(AsmArgs a) {
  const eaf_assembly_fields_t& f = a.f;
  for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < a.nh;
       q += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_of(a, q, i, j, k);
    if (i < 1 || i > a.nr + 1 || j < 1 || j > a.nth + 1 || k < 1 || k > a.nz + 1) continue;
    LowerFaces L;
    L.q = q;
    L.x[0] = q - 1;
    L.x[1] = q - a.sx;
    L.x[2] = q - a.sxy;
    const unsigned cell[4] = {q, L.x[0], L.x[1], L.x[2]};
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      L.ct[m] = ld(f.cell_type, cell[m]);
      L.p[m] = ld(f.p, cell[m]);
      L.vol[m] = ld(f.vol, cell[m]);
      L.room[m] = ROOM ? ld(f.liq_room, cell[m]) : 1.0;
    }
    const double r0 = ld(f.r, i), r1 = ld(f.r, i + 1);
    const double t0 = ld(f.theta, j), t1 = ld(f.theta, j + 1);
    const double z0 = ld(f.z, k), z1 = ld(f.z, k + 1);
    L.delta[0] = r1 - r0;
    L.delta[1] = r1 * (t1 - t0);
    L.delta[2] = z1 - z0;
    L.area[0] = ld(f.Ar, L.x[0]);
    L.area[1] = 0.0;
    L.area[2] = ld(f.Az, L.x[2]);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      L.ok[m] = exp_in_safe_range(L.delta[m]);
      L.y[m] = L.ok[m] ? 1.0 / L.delta[m] : 0.0;
      // + side minus - side
      L.gp[m] = div_by_recip(L.p[0] - L.p[m + 1], L.delta[m], L.y[m], L.ok[m]);
    }
    unsigned bits = phase_faces<false, ROOM>(a, L, f.liq, f.act_l, a.gz_l, 0.0, a.fl);
    if (GAS_IN) {
      // liquid weight of the B face (liq_weight_f :407-417, lower cell first)
      const unsigned b = L.x[2];
      const double lw_b = liq_weight(f.beta_expansion, f.T_ambient, ld(f.act_l, b) != 0,
                                     ld(f.liq.alpha, b), ld(f.liq.rho, b), ld(f.liq_T, b),
                                     ld(f.act_l, q) != 0, ld(f.liq.alpha, q),
                                     ld(f.liq.rho, q), ld(f.liq_T, q));
      bits |= phase_faces<true, false>(a, L, f.gas, f.act_g, a.gz_g, lw_b, a.fg) << kGasShift;
    }
    a.open[q] = (unsigned char)bits;
  }
}

struct CellOut {
  double aW, aE, aS, aN, aB, aT, aP, Su;
  double Fs_r, Fs_th, Fs_z, ac_r, ac_th, ac_z;
  int lk_r, lk_th, lk_z;
  double flux;
};

// Face values of one phase that cell q adds: its own W, S, B faces and the
// W, S, B faces of e, n, t (its E, N, T faces).
struct FaceVals {
  double cW, fW, cE, fE, aS, uS, aN, uN, cB, fB, cT, fT;
};

__device__ __forceinline__ void load_faces(const FacePhase& F, unsigned q, unsigned e,
                                           unsigned n, unsigned t, FaceVals& v) {
  v.cW = ld(F.cW, q); v.fW = ld(F.fW, q); v.cE = ld(F.cW, e); v.fE = ld(F.fW, e);
  v.aS = ld(F.dS, q); v.uS = ld(F.uS, q); v.aN = ld(F.dS, n); v.uN = ld(F.uS, n);
  v.cB = ld(F.cB, q); v.fB = ld(F.fB, q); v.cT = ld(F.cB, t); v.fT = ld(F.fB, t);
}

// The six faces of one phase at cell q, added in the reference's order
// W, E, S, N, B, T; theta faces take this cell's area. bq, be, bn, bt are
// the open bits of q, e, n, t for this phase.
template <bool EXPORT>
__device__ __forceinline__ void add_faces(const FaceVals& v, unsigned bq, unsigned be,
                                          unsigned bn, unsigned bt, double Ath, double dS,
                                          double yS, bool okS, double dN, double yN, bool okN,
                                          CellOut& o) {
  const double cS = div_by_recip(v.aS * Ath, dS, yS, okS), fS = v.uS * Ath;
  const double cN = div_by_recip(v.aN * Ath, dN, yN, okN), fN = v.uN * Ath;
  if (bq & kBitW) {
    o.aW = o.aW + v.cW;
    o.Su = o.Su + v.fW;
    o.flux = o.flux + fabs(v.fW);
  }
  if (be & kBitW) {
    o.aE = o.aE + v.cE;
    o.Su = o.Su - v.fE;
    o.flux = o.flux + fabs(v.fE);
    if (EXPORT) { o.Fs_r = v.fE; o.ac_r = v.cE; o.lk_r = 1; }
  }
  if (bq & kBitS) {
    o.aS = o.aS + cS;
    o.Su = o.Su + fS;
    o.flux = o.flux + fabs(fS);
  }
  if (bn & kBitS) {
    o.aN = o.aN + cN;
    o.Su = o.Su - fN;
    o.flux = o.flux + fabs(fN);
    if (EXPORT) { o.Fs_th = fN; o.ac_th = cN; o.lk_th = 1; }
  }
  if (bq & kBitB) {
    o.aB = o.aB + v.cB;
    o.Su = o.Su + v.fB;
    o.flux = o.flux + fabs(v.fB);
  }
  if (bt & kBitB) {
    o.aT = o.aT + v.cT;
    o.Su = o.Su - v.fT;
    o.flux = o.flux + fabs(v.fT);
    if (EXPORT) { o.Fs_z = v.fT; o.ac_z = v.cT; o.lk_z = 1; }
  }
}

template <bool GAS_IN, bool GAS_COMP>
__global__ void __launch_bounds__(kAsmBlock, 2) asm_cell_kernel(AsmArgs a) {
  const eaf_assembly_fields_t& f = a.f;
  double v[2] = {0.0, 0.0};  // flux_ref, sum |Su|
  for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < a.nh;
       q += gridDim.x * blockDim.x) {
    CellOut o = {};
    int i, j, k;
    cell_of(a, q, i, j, k);
    const bool inner = i >= 1 && i <= a.nr && j >= 1 && j <= a.nth && k >= 1 && k <= a.nz;
    if (inner) {
      const Stencil st(q, a.sx, a.sxy);
      // outlets count on the top layer only: read for cells on it (their
      // own and w, e, s, n) and just below it (t)
      const bool top = k == a.nz, below_top = k == a.nz - 1;
      int ct[7], ot[7];
#pragma unroll
      for (int m = 0; m < 7; ++m) {
        ct[m] = ld(f.cell_type, st.q[m]);
        const bool on_top = m == T ? below_top : (m != B && top);
        ot[m] = on_top ? ld(f.outlet, st.q[m]) : 0;
      }
      const int l_act = ld(f.act_l, q), g_act = ld(f.act_g, q);
      const unsigned e = st.q[E], n = st.q[N], t = st.q[T];
      const unsigned bq = ld(a.open, q), be = ld(a.open, e), bn = ld(a.open, n),
                     bt = ld(a.open, t);
      const double vol = ld(f.vol, q), Ath = ld(f.Ath, q);
      const double r1 = ld(f.r, i + 1);
      const double t0 = ld(f.theta, j), t1 = ld(f.theta, j + 1), t2 = ld(f.theta, j + 2);
      const double la = ld(f.liq.alpha, q), lr = ld(f.liq.rho, q);
      double ga = 0.0, gr = 0.0, gT = 0.0;
      if (GAS_COMP) {
        ga = ld(f.gas.alpha, q);
        gr = ld(f.gas.rho, q);
        gT = ld(f.gas_T_old, q);
      }

      if (ct[C] != 0) {
        const bool l_on = l_act != 0, g_on = g_act != 0;
        const double dS = r1 * (t1 - t0), dN = r1 * (t2 - t1);
        const bool okS = exp_in_safe_range(dS), okN = exp_in_safe_range(dN);
        const double yS = okS ? 1.0 / dS : 0.0, yN = okN ? 1.0 / dN : 0.0;
        FaceVals fv;
        if (l_on) {
          load_faces(a.fl, q, e, n, t, fv);
          add_faces<true>(fv, bq, be, bn, bt, Ath, dS, yS, okS, dN, yN, okN, o);
        }
        if (GAS_IN && g_on) {
          load_faces(a.fg, q, e, n, t, fv);
          add_faces<false>(fv, bq >> kGasShift, be >> kGasShift, bn >> kGasShift,
                           bt >> kGasShift, Ath, dS, yS, okS, dN, yN, okN, o);
        }
        if (GAS_COMP && g_on) {  // (:228-247)
          const double src = ga * vol / f.dt *
                             (gr - f.rho_gas * f.T_ambient / fmax(gT, kTminGas)) /
                             fmax(gr, kS);
          const double cap = kCompCap * ga * vol / f.dt;
          o.Su = o.Su - fmax(-cap, fmin(cap, src));
        }
        if (!l_on && !g_on) {  // (:253-259)
          o.aW = 0.0; o.aE = 0.0; o.aS = 0.0; o.aN = 0.0; o.aB = 0.0; o.aT = 0.0;
          o.aP = 1.0; o.Su = 0.0;
        } else {  // (:260-283)
          o.aP = (o.aW + o.aE + o.aS + o.aN + o.aB + o.aT) * (1.0 + kCompliance);
          if (GAS_COMP && g_on) o.aP = o.aP + ga / kP0 * vol / f.dt;
          if (l_on) o.aP = o.aP + la * vol / (lr * (kCsound * kCsound) * f.dt);
        }
        // apply_pressure_bc (serial: every boundary physical); out[m] = stencil
        // cell m is an electrode hole of the top layer
        bool out[7];
#pragma unroll
        for (int m = 0; m < 7; ++m) out[m] = ot[m] != 0;
        if (i == 1) o.aW = 0.0;
        if (i == a.nr) o.aE = 0.0;
        if (k == 1) o.aB = 0.0;
        if (out[C]) {
          o.aW = 0.0; o.aE = 0.0; o.aS = 0.0; o.aN = 0.0; o.aB = 0.0; o.aT = 0.0;
          o.aP = 1.0; o.Su = 0.0;
        } else {
          if (top) o.aT = 0.0;
          if (i > 1 && ct[W] == 0) o.aW = 0.0;
          if (i < a.nr && ct[E] == 0) o.aE = 0.0;
          if (k > 1 && ct[B] == 0) o.aB = 0.0;
          if (k < a.nz && ct[T] == 0) o.aT = 0.0;
          if (out[W]) o.aW = 0.0;
          if (out[E]) o.aE = 0.0;
          if (out[S]) o.aS = 0.0;
          if (out[N]) o.aN = 0.0;
          if (out[T]) o.aT = 0.0;  // b always lies below the top layer
        }
        v[0] = v[0] + o.flux;
        if (l_on || g_on) v[1] = v[1] + fabs(o.Su);
      } else {  // solid cell: identity row (apply_pressure_bc)
        o.aP = 1.0;
      }
    }
    f.aW[q] = o.aW; f.aE[q] = o.aE; f.aS[q] = o.aS; f.aN[q] = o.aN;
    f.aB[q] = o.aB; f.aT[q] = o.aT; f.aP[q] = o.aP; f.Su[q] = o.Su;
    f.pp[q] = 0.0;
    f.Fs_r[q] = o.Fs_r; f.Fs_th[q] = o.Fs_th; f.Fs_z[q] = o.Fs_z;
    f.ac_r[q] = o.ac_r; f.ac_th[q] = o.ac_th; f.ac_z[q] = o.ac_z;
    f.Fc_r[q] = 0.0; f.Fc_th[q] = 0.0; f.Fc_z[q] = 0.0;
    f.lk_r[q] = o.lk_r; f.lk_th[q] = o.lk_th; f.lk_z[q] = o.lk_z;
  }
  block_sum_to_thread0<2, double>(v);
  if (threadIdx.x == 0) {
    a.part[blockIdx.x] = v[0];
    a.part[gridDim.x + blockIdx.x] = v[1];
  }
}

// One block: thread t sums block partials t, t + blockDim, ... in order, then
// a fixed-order block reduction; residual = sum_su / max(flux_ref, SMALL)
// (:305). Deterministic for a given grid.
constexpr int kAsmResBlock = 1024;
__global__ void __launch_bounds__(kAsmResBlock) asm_residual_kernel(AsmArgs a, int nblocks) {
  double s[2] = {0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    s[0] = s[0] + a.part[b];
    s[1] = s[1] + a.part[nblocks + b];
  }
  block_sum_to_thread0<2, double>(s);
  if (threadIdx.x == 0) *a.result = s[1] / fmax(s[0], kS);
}

unsigned asm_grid(long long work) {
  long long g = (work + kAsmBlock - 1) / kAsmBlock;
  if (g < 1) g = 1;
  if (g > 148 * 8) g = 148 * 8;
  return (unsigned)g;
}

}  // namespace

// Scratch: 4 gradient arrays, 12 face arrays (6 per phase), the open bits,
// the block partials and the residual.
size_t assembly_scratch_doubles(int nr, int nth, int nz) {
  const size_t nh = (size_t)(nr + 4) * (nth + 4) * (nz + 4);
  return 16 * nh + (nh + 7) / 8 + 2 * 148 * 8 + 1;
}

cudaError_t launch_assemble_f64(const eaf_assembly_fields_t& f, int nr, int nth, int nz,
                                double* scratch, cudaStream_t st) {
  AsmArgs a;
  a.f = f;
  a.nr = nr;
  a.nth = nth;
  a.nz = nz;
  a.sx = (unsigned)(nr + 4);
  a.rows = (unsigned)(nth + 4);
  a.sxy = a.sx * a.rows;
  a.nh = a.sxy * (unsigned)(nz + 4);
  double* w = scratch;
  auto take = [&](size_t n) { double* r = w; w += n; return r; };
  a.gr = take(a.nh);
  a.gth = take(a.nh);
  a.gz_l = take(a.nh);
  a.gz_g = take(a.nh);
  for (FacePhase* F : {&a.fl, &a.fg}) {
    F->cW = take(a.nh);
    F->fW = take(a.nh);
    F->dS = take(a.nh);
    F->uS = take(a.nh);
    F->cB = take(a.nh);
    F->fB = take(a.nh);
  }
  a.open = reinterpret_cast<unsigned char*>(take((a.nh + 7) / 8));
  const unsigned gf = asm_grid(a.nh);
  a.part = take(2 * gf);
  a.result = take(1);
  const bool gi = f.gas_in_poisson != 0, gc = f.gas_compressibility != 0,
             rm = f.liq_room_valid != 0;
  if (gi) asm_gradient_kernel<true><<<gf, kAsmBlock, 0, st>>>(a);
  else asm_gradient_kernel<false><<<gf, kAsmBlock, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  using K = void (*)(AsmArgs);
  const K faces[4] = {asm_face_kernel<false, false>, asm_face_kernel<false, true>,
                      asm_face_kernel<true, false>, asm_face_kernel<true, true>};
  faces[(gi ? 2 : 0) + (rm ? 1 : 0)]<<<gf, kAsmBlock, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const K cells[4] = {asm_cell_kernel<false, false>, asm_cell_kernel<false, true>,
                      asm_cell_kernel<true, false>, asm_cell_kernel<true, true>};
  cells[(gi ? 2 : 0) + (gc ? 1 : 0)]<<<gf, kAsmBlock, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  asm_residual_kernel<<<1, kAsmResBlock, 0, st>>>(a, (int)gf);
  return cudaGetLastError();
}

const double* assembly_result(double* scratch, int nr, int nth, int nz) {
  const size_t nh = (size_t)(nr + 4) * (nth + 4) * (nz + 4);
  return scratch + 16 * nh + (nh + 7) / 8 + 2 * (size_t)asm_grid((long long)nh);
}

}  // namespace eaf
