// Assembly of the pressure-correction equation on the device: the serial
// code of solve_pressure_correction before the CG (src/mod_pressure_3d.f90:
// 135-310). Three launches:
//   G. cell gradients (cell_gradients :621-651) of the liquid and, for the
//      gas, the vertical one with the liquid weight (gas_gz :421-440; its r
//      and theta gradients equal the liquid's); one thread per halo element,
//      theta halo rows computing their source row of the periodic copy, so
//      neither a clearing pass nor a halo pass is needed;
//   F. one thread per halo element: every output zeroed, and in interior
//      cells the face contributions of the liquid then the gas
//      (add_phase_contribution :469-619), the compressibility source
//      (:228-247), trivial rows and the diagonal (:250-285) and the boundary
//      folding (apply_pressure_bc, src/mod_boundary_3d.f90:180-277), all in
//      the reference's per-cell order -- each cell only reads inputs and the
//      gradients; per-block partials of flux_ref and sum |Su|;
//   R. the block partials folded in a fixed order into the residual.
// Built with -fmad=false, like the other units that must match the
// reference's non-FMA arithmetic.
#include <cuda_runtime.h>
#include <stdint.h>

#include "cg_common.cuh"
#include "cg_kernels.h"
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

struct AsmArgs {
  eaf_assembly_fields_t f;
  double *gr, *gth, *gz_l, *gz_g;  // gradient scratch (halo layout)
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
__global__ void __launch_bounds__(kAsmBlock) asm_gradient_kernel(AsmArgs a) {
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

struct CellOut {
  double aW, aE, aS, aN, aB, aT, aP, Su;
  double Fs_r, Fs_th, Fs_z, ac_r, ac_th, ac_z;
  int lk_r, lk_th, lk_z;
  double flux;
};

// Shared per-cell inputs of both phases.
struct CellIn {
  Stencil st;
  int i, j, k;
  int ct[7];
  double p[7], vol[7], room[7];
  double r0, r1, r2, t0, t1, t2, z0, z1, z2;
  double Ar_w, Ar_c, Ath_c, Az_b, Az_c;
  __device__ CellIn(unsigned q, unsigned sx, unsigned sxy) : st(q, sx, sxy) {}
};

// face_open (:660-668)
template <bool ISG, bool ROOM>
__device__ __forceinline__ bool face_open(double u_f, double room_neg, double room_pos) {
  if (ISG || !ROOM) return true;
  bool open = true;
  if (u_f > 0.0 && room_pos <= kRoomEps) open = false;
  if (u_f < 0.0 && room_neg <= kRoomEps) open = false;
  return open;
}

// add_phase_contribution (:469-619) at an interior cell whose phase is
// active; lk[m] = the phase links to stencil cell m; gas faces add the
// liquid weight lw_b / lw_t to the vertical ones. The six faces are computed
// without branches, in one block (their divisions independent of each
// other), and added in the reference's order W, E, S, N, B, T where linked
// and open; the arithmetic of each face is the reference's (sums of two
// terms commute exactly, and subtracting a zero weight is exact).
template <bool ISG, bool ROOM, bool EXPORT>
__device__ __forceinline__ void add_phase(const CellIn& c, const eaf_phase_state_t& ph,
                                          const double* gr, const double* gth,
                                          const double* gz, const bool lk[7], double lw_b,
                                          double lw_t, CellOut& o) {
  const unsigned* q = c.st.q;
  double al[7];
#pragma unroll
  for (int m = 0; m < 7; ++m) al[m] = ld(ph.alpha, q[m]);
  // per face f = 0..5 (W, E, S, N, B, T): stencil cell f + 1, direction f / 2
  const double* apd[3] = {ph.aP_ur, ph.aP_uth, ph.aP_uz};
  const double* ud[3] = {ph.ur, ph.uth, ph.uz};
  const double* gd[3] = {gr, gth, gz};
  double ap_c[3], u_c[3], g_c[3], ap_x[6], u_x[6], g_x[6];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ap_c[d] = ld(apd[d], q[C]);
    u_c[d] = ld(ud[d], q[C]);
    g_c[d] = ld(gd[d], q[C]);
  }
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    ap_x[f] = ld(apd[f / 2], q[f + 1]);
    u_x[f] = ld(ud[f / 2], q[f + 1]);
    g_x[f] = ld(gd[f / 2], q[f + 1]);
  }
  const double* p = c.p;
  const double* vol = c.vol;
  const double* rm = c.room;
  const double delta[6] = {c.r1 - c.r0,          c.r2 - c.r1,          c.r1 * (c.t1 - c.t0),
                           c.r1 * (c.t2 - c.t1), c.z1 - c.z0,          c.z2 - c.z1};
  // pressure difference across the face, + side minus - side
  const double dp[6] = {p[C] - p[W], p[E] - p[C], p[C] - p[S],
                        p[N] - p[C], p[C] - p[B], p[T] - p[C]};
  const double area[6] = {c.Ar_w, c.Ar_c, c.Ath_c, c.Ath_c, c.Az_b, c.Az_c};
  const double lw[6] = {0.0, 0.0, 0.0, 0.0, lw_b, lw_t};
  double ctm[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) ctm[d] = al[C] * vol[C] / fmax(ap_c[d], kS);
  double coef[6], flux[6];
  bool open[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int x = f + 1, d = f / 2;
    const double d_f = 0.5 * (ctm[d] + al[x] * vol[x] / fmax(ap_x[f], kS));
    const double af = 0.5 * (al[C] + al[x]);
    const double u_f = 0.5 * (u_c[d] + u_x[f]) +
                       d_f * (0.5 * (g_c[d] + g_x[f]) - dp[f] / delta[f] - lw[f]);
    // the face's - side and + side rooms
    const bool lower = (f & 1) == 0;
    open[f] = lk[x] && face_open<ISG, ROOM>(u_f, lower ? rm[x] : rm[C], lower ? rm[C] : rm[x]);
    coef[f] = af * d_f * area[f] / delta[f];
    flux[f] = af * u_f * area[f];
  }
  double* acc[6] = {&o.aW, &o.aE, &o.aS, &o.aN, &o.aB, &o.aT};
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (open[f]) {
      *acc[f] = *acc[f] + coef[f];
      o.Su = (f & 1) == 0 ? o.Su + flux[f] : o.Su - flux[f];
      o.flux = o.flux + fabs(flux[f]);
    }
  }
  if (EXPORT) {
    if (open[1]) { o.Fs_r = flux[1]; o.ac_r = coef[1]; o.lk_r = 1; }
    if (open[3]) { o.Fs_th = flux[3]; o.ac_th = coef[3]; o.lk_th = 1; }
    if (open[5]) { o.Fs_z = flux[5]; o.ac_z = coef[5]; o.lk_z = 1; }
  }
}

template <bool GAS_IN, bool GAS_COMP, bool ROOM>
__global__ void __launch_bounds__(kAsmBlock) asm_face_kernel(AsmArgs a) {
  const eaf_assembly_fields_t& f = a.f;
  double v[2] = {0.0, 0.0};  // flux_ref, sum |Su|
  for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < a.nh;
       q += gridDim.x * blockDim.x) {
    CellOut o = {};
    CellIn c(q, a.sx, a.sxy);
    cell_of(a, q, c.i, c.j, c.k);
    const bool inner = c.i >= 1 && c.i <= a.nr && c.j >= 1 && c.j <= a.nth && c.k >= 1 &&
                       c.k <= a.nz;
    if (inner) {
      int al[7], ag[7];
      // outlets count on the top layer only: read for cells on it (their
      // own and w, e, s, n) and just below it (t)
      const bool top = c.k == a.nz, below_top = c.k == a.nz - 1;
      int ot[7];
#pragma unroll
      for (int m = 0; m < 7; ++m) {
        c.ct[m] = ld(f.cell_type, c.st.q[m]);
        al[m] = ld(f.act_l, c.st.q[m]);
        ag[m] = ld(f.act_g, c.st.q[m]);
        const bool on_top = m == T ? below_top : (m != B && top);
        ot[m] = on_top ? ld(f.outlet, c.st.q[m]) : 0;
        c.p[m] = ld(f.p, c.st.q[m]);
        c.vol[m] = ld(f.vol, c.st.q[m]);
        c.room[m] = ROOM ? ld(f.liq_room, c.st.q[m]) : 1.0;
      }
      c.r0 = ld(f.r, c.i); c.r1 = ld(f.r, c.i + 1); c.r2 = ld(f.r, c.i + 2);
      c.t0 = ld(f.theta, c.j); c.t1 = ld(f.theta, c.j + 1); c.t2 = ld(f.theta, c.j + 2);
      c.z0 = ld(f.z, c.k); c.z1 = ld(f.z, c.k + 1); c.z2 = ld(f.z, c.k + 2);
      c.Ar_w = ld(f.Ar, c.st.q[W]);
      c.Ar_c = ld(f.Ar, q);
      c.Ath_c = ld(f.Ath, q);
      c.Az_b = ld(f.Az, c.st.q[B]);
      c.Az_c = ld(f.Az, q);
      if (c.ct[C] != 0) {
        const bool l_on = al[C] != 0, g_on = ag[C] != 0;
        bool lk[7];
        if (l_on) {
#pragma unroll
          for (int m = 0; m < 7; ++m) lk[m] = (c.ct[m] != 0) & (al[m] != 0);
          add_phase<false, ROOM, true>(c, f.liq, a.gr, a.gth, a.gz_l, lk, 0.0, 0.0, o);
        }
        if (GAS_IN && g_on) {
          // liquid weights of the two vertical faces
          double la[3], lr[3], lT[3];
          const int cbt[3] = {C, B, T};
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            la[m] = ld(f.liq.alpha, c.st.q[cbt[m]]);
            lr[m] = ld(f.liq.rho, c.st.q[cbt[m]]);
            lT[m] = ld(f.liq_T, c.st.q[cbt[m]]);
          }
          const double beta = f.beta_expansion, ta = f.T_ambient;
          const double lw_b = liq_weight(beta, ta, al[B] != 0, la[1], lr[1], lT[1],
                                         al[C] != 0, la[0], lr[0], lT[0]);
          const double lw_t = liq_weight(beta, ta, al[C] != 0, la[0], lr[0], lT[0],
                                         al[T] != 0, la[2], lr[2], lT[2]);
#pragma unroll
          for (int m = 0; m < 7; ++m) lk[m] = (c.ct[m] != 0) & (ag[m] != 0);
          add_phase<true, false, false>(c, f.gas, a.gr, a.gth, a.gz_g, lk, lw_b, lw_t, o);
        }
        double ag_alpha = 0.0;
        if (GAS_COMP && g_on) {  // (:228-247)
          ag_alpha = ld(f.gas.alpha, q);
          const double vo = c.vol[C], rh = ld(f.gas.rho, q), Told = ld(f.gas_T_old, q);
          const double src = ag_alpha * vo / f.dt *
                             (rh - f.rho_gas * f.T_ambient / fmax(Told, kTminGas)) /
                             fmax(rh, kS);
          const double cap = kCompCap * ag_alpha * vo / f.dt;
          o.Su = o.Su - fmax(-cap, fmin(cap, src));
        }
        if (!l_on && !g_on) {  // (:253-259)
          o.aW = 0.0; o.aE = 0.0; o.aS = 0.0; o.aN = 0.0; o.aB = 0.0; o.aT = 0.0;
          o.aP = 1.0; o.Su = 0.0;
        } else {  // (:260-283)
          o.aP = (o.aW + o.aE + o.aS + o.aN + o.aB + o.aT) * (1.0 + kCompliance);
          if (GAS_COMP && g_on) o.aP = o.aP + ag_alpha / kP0 * c.vol[C] / f.dt;
          if (l_on)
            o.aP = o.aP + ld(f.liq.alpha, q) * c.vol[C] /
                              (ld(f.liq.rho, q) * (kCsound * kCsound) * f.dt);
        }
        // apply_pressure_bc (serial: every boundary physical); out[m] = stencil
        // cell m is an electrode hole of the top layer
        bool out[7];
#pragma unroll
        for (int m = 0; m < 7; ++m) out[m] = ot[m] != 0;
        if (c.i == 1) o.aW = 0.0;
        if (c.i == a.nr) o.aE = 0.0;
        if (c.k == 1) o.aB = 0.0;
        if (out[C]) {
          o.aW = 0.0; o.aE = 0.0; o.aS = 0.0; o.aN = 0.0; o.aB = 0.0; o.aT = 0.0;
          o.aP = 1.0; o.Su = 0.0;
        } else {
          if (top) o.aT = 0.0;
          if (c.i > 1 && c.ct[W] == 0) o.aW = 0.0;
          if (c.i < a.nr && c.ct[E] == 0) o.aE = 0.0;
          if (c.k > 1 && c.ct[B] == 0) o.aB = 0.0;
          if (c.k < a.nz && c.ct[T] == 0) o.aT = 0.0;
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

// One warp: lane l sums block partials l, l+32, ... in order, then the
// butterfly; residual = sum_su / max(flux_ref, SMALL) (:305).
__global__ void asm_residual_kernel(AsmArgs a, int nblocks) {
  double s[2];
  for (int m = 0; m < 2; ++m) {
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 32) acc = acc + a.part[m * nblocks + b];
    s[m] = warp_allsum(acc);
  }
  if (threadIdx.x == 0) *a.result = s[1] / fmax(s[0], kS);
}

unsigned asm_grid(long long work) {
  long long g = (work + kAsmBlock - 1) / kAsmBlock;
  if (g < 1) g = 1;
  if (g > 148 * 8) g = 148 * 8;
  return (unsigned)g;
}

}  // namespace

size_t assembly_scratch_doubles(int nr, int nth, int nz) {
  return (size_t)4 * (nr + 4) * (nth + 4) * (nz + 4) + 2 * 148 * 8 + 1;
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
  a.gr = scratch;
  a.gth = a.gr + a.nh;
  a.gz_l = a.gth + a.nh;
  a.gz_g = a.gz_l + a.nh;
  a.part = a.gz_g + a.nh;
  const unsigned gf = asm_grid(a.nh);
  a.result = a.part + 2 * gf;
  const bool gi = f.gas_in_poisson != 0, gc = f.gas_compressibility != 0,
             rm = f.liq_room_valid != 0;
  if (gi) asm_gradient_kernel<true><<<gf, kAsmBlock, 0, st>>>(a);
  else asm_gradient_kernel<false><<<gf, kAsmBlock, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  using K = void (*)(AsmArgs);
  const K faces[8] = {asm_face_kernel<false, false, false>, asm_face_kernel<false, false, true>,
                      asm_face_kernel<false, true, false>,  asm_face_kernel<false, true, true>,
                      asm_face_kernel<true, false, false>,  asm_face_kernel<true, false, true>,
                      asm_face_kernel<true, true, false>,   asm_face_kernel<true, true, true>};
  faces[(gi ? 4 : 0) + (gc ? 2 : 0) + (rm ? 1 : 0)]<<<gf, kAsmBlock, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  asm_residual_kernel<<<1, 32, 0, st>>>(a, (int)gf);
  return cudaGetLastError();
}

const double* assembly_result(double* scratch, int nr, int nth, int nz) {
  const long long nh = (long long)(nr + 4) * (nth + 4) * (nz + 4);
  const long long gf = asm_grid(nh);
  return scratch + 4 * nh + 2 * gf;
}

}  // namespace eaf
