// Post-CG corrections of the pressure-correction step on the device: the
// serial code after the CG in solve_pressure_correction
// (src/mod_pressure_3d.f90:333-397) and correct_velocities (:689-746).
//
// Every step reads the CG solution pp and writes arrays that no other step
// of the same kernel reads, except the sealed-cell rule, which reads the
// updated p of ACTIVE neighbours and writes SEALED cells only; so three
// launches reproduce the sequential loops exactly:
//   1. one pass over the whole halo array: p = clamp(p + alpha_p pp) for
//      every element; in interior non-solid cells the face fluxes and the
//      velocity corrections of both phases;
//   2. the sealed-cell mean over the updated p;
//   3. the theta-halo refresh of Fc_r/th/z, lk_r/th/z and p.
// All HBM-bound streaming; built with -fmad=false so every a*b+c rounds
// twice, as the reference's non-FMA build does.
#include <cuda_runtime.h>
#include <stdint.h>

#include "cg_kernels.h"
#include "eafcg.h"

namespace eaf {
namespace {

constexpr double kSmallP = 1.0e-30;   // SMALL, src/mod_constants.f90:53
constexpr double kHydroCap = 2.0e6;   // P_HYDRO_CAP, src/mod_pressure_3d.f90:79

struct PcorrArgs {
  eaf_pcorr_fields_t f;
  int nr, nth, nz;
  long long sx, sxy, nh;
};

// correct_velocities (src/mod_pressure_3d.f90:711-742) of one phase at one
// interior cell, from values already in registers: pp neighbours
// (ppE/ppW along r, ppN/ppS along theta, ppT/ppB along z) and the cell's
// coordinate differences; returns the corrected velocities.
struct CellGeo {
  double pp_e, pp_w, pp_n, pp_s, pp_t, pp_b;
  double dr2, rth2, dz2;  // r(i+1)-r(i-1), r(i)*(theta(j+1)-theta(j-1)), z(k+1)-z(k-1)
  double vol;
  bool skip_r, skip_z;
};

struct PhaseVals {
  double alpha, aur, auth, auz, ur, uth, uz;
};

__device__ __forceinline__ PhaseVals load_phase(const eaf_phase_fields_t& ph, long long q) {
  PhaseVals v;
  v.alpha = ph.alpha[q];
  v.aur = ph.aP_ur[q];
  v.auth = ph.aP_uth[q];
  v.auz = ph.aP_uz[q];
  v.ur = ph.ur[q];
  v.uth = ph.uth[q];
  v.uz = ph.uz[q];
  return v;
}

__device__ __forceinline__ void correct_phase(PhaseVals& v, const CellGeo& c) {
  if (!c.skip_r && fabs(v.aur) > kSmallP) {
    const double dc = v.alpha * c.vol / v.aur;
    v.ur = v.ur - dc * (c.pp_e - c.pp_w) / c.dr2;
  }
  if (fabs(v.auth) > kSmallP) {
    const double dc = v.alpha * c.vol / v.auth;
    v.uth = v.uth - dc * (c.pp_n - c.pp_s) / c.rth2;
  }
  if (!c.skip_z && fabs(v.auz) > kSmallP) {
    const double dc = v.alpha * c.vol / v.auz;
    v.uz = v.uz - dc * (c.pp_t - c.pp_b) / c.dz2;
  }
}

// One pass over the whole halo array, every load issued before any branch
// (halo elements load their own entries in place of neighbours and an
// interior coordinate, then write only p): p = clamp(p + alpha_p pp)
// everywhere (:358-360); in interior non-solid cells the face fluxes
// (:333-345) and the velocity corrections of both phases (:354-356).
__global__ void __launch_bounds__(256) pcorr_update_kernel(PcorrArgs a) {
  // Lets the next launch of the chain be scheduled early; it waits for this
  // grid's completion (griddepcontrol.wait) before touching memory.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const eaf_pcorr_fields_t& f = a.f;
  const long long rows = a.nth + 4;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < a.nh;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % a.sx) - 1;
    const long long t = q / a.sx;
    const int j = (int)(t % rows) - 1, k = (int)(t / rows) - 1;
    const bool inner = i >= 1 && i <= a.nr && j >= 1 && j <= a.nth && k >= 1 && k <= a.nz;
    const long long o1 = inner ? 1 : 0, osx = inner ? a.sx : 0, osxy = inner ? a.sxy : 0;
    const int ci = inner ? i : 1, cj = inner ? j : 1, ck = inner ? k : 1;
    const double* pp = f.pp;
    const double ppc = pp[q], pv0 = f.p[q];
    CellGeo g;
    g.pp_e = pp[q + o1];
    g.pp_w = pp[q - o1];
    g.pp_n = pp[q + osx];
    g.pp_s = pp[q - osx];
    g.pp_t = pp[q + osxy];
    g.pp_b = pp[q - osxy];
    const int ct = f.cell_type[q];
    const int lr = f.lk_r[q], lt = f.lk_th[q], lz = f.lk_z[q];
    const int al = f.act_l[q], ag = f.act_g[q];
    const double fsr = f.Fs_r[q], fst = f.Fs_th[q], fsz = f.Fs_z[q];
    const double acr = f.ac_r[q], act = f.ac_th[q], acz = f.ac_z[q];
    g.vol = f.vol[q];
    const double r_p = f.r[ci + 2], r_m = f.r[ci], r_c = f.r[ci + 1];
    const double th_p = f.theta[cj + 2], th_m = f.theta[cj];
    const double z_p = f.z[ck + 2], z_m = f.z[ck];
    PhaseVals liq = load_phase(f.liq, q);
    PhaseVals gas;
    if (f.has_gas) gas = load_phase(f.gas, q);
    // p over the whole array
    const double pv = pv0 + f.alpha_p * ppc;
    f.p[q] = fmax(-kHydroCap, fmin(kHydroCap, pv));
    if (!inner || ct == 0) continue;
    if (lr == 1) f.Fc_r[q] = fsr + acr * (ppc - g.pp_e);
    if (lt == 1) f.Fc_th[q] = fst + act * (ppc - g.pp_n);
    if (lz == 1) f.Fc_z[q] = fsz + acz * (ppc - g.pp_t);
    g.dr2 = r_p - r_m;
    g.rth2 = r_c * (th_p - th_m);
    g.dz2 = z_p - z_m;
    g.skip_r = (i == 1) || (i == a.nr);
    g.skip_z = (k == 1) || (k == a.nz);
    if (al) {
      correct_phase(liq, g);
      f.liq.ur[q] = liq.ur;
      f.liq.uth[q] = liq.uth;
      f.liq.uz[q] = liq.uz;
    }
    if (f.has_gas && ag) {
      correct_phase(gas, g);
      f.gas.ur[q] = gas.ur;
      f.gas.uth[q] = gas.uth;
      f.gas.uz[q] = gas.uz;
    }
  }
}

// (:373-395) with acc_nb (:451-458): neighbours in the order i-1, i+1,
// j-1, j+1, k-1, k+1, summed from 0. The cell's own flags come first in one
// round of loads; only sealed cells (a few per cent) read their neighbours.
__global__ void pcorr_sealed_kernel(PcorrArgs a) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // the updated p of the previous launch, complete and visible
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const eaf_pcorr_fields_t& f = a.f;
  const long long n = (long long)a.nr * a.nth * a.nz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % a.nr) + 1;
    const long long t = c / a.nr;
    const int j = (int)(t % a.nth) + 1, k = (int)(t / a.nth) + 1;
    const long long q = (long long)(i + 1) + a.sx * (j + 1) + a.sxy * (k + 1);
    const int ct = f.cell_type[q], al = f.act_l[q], ag = f.act_g[q];
    if (ct == 0 || al || ag) continue;
    const long long nb[6] = {q - 1, q + 1, q - a.sx, q + a.sx, q - a.sxy, q + a.sxy};
    int nct[6], nal[6], nag[6];
    double np[6];
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      nct[u] = f.cell_type[nb[u]];
      nal[u] = f.act_l[nb[u]];
      nag[u] = f.act_g[nb[u]];
      np[u] = f.p[nb[u]];
    }
    double psum = 0.0;
    int nnb = 0;
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      if (nct[u] == 0) continue;
      if (!nal[u] && !nag[u]) continue;
      psum = psum + np[u];
      nnb = nnb + 1;
    }
    f.p[q] = nnb > 0 ? psum / (double)nnb : 0.0;
  }
}

// Serial theta-periodic copy (src/mod_mpi_topology.f90:303-311 and its int
// twin :686-692) of one (i, k) column of x. The four sources are read before
// any store: with nth >= 2 no source is a destination, and with nth == 1
// the second and fourth statements read what the first and third wrote --
// the values of columns nth and 1 -- so the result is the sequential one.
template <typename T>
__device__ __forceinline__ void wrap_column(T* x, long long col_base, long long sx, int nth) {
  T* p = x + col_base;
  auto J = [&](int j) { return (long long)(j + 1) * sx; };
  const T v0 = p[J(nth)];
  const T v1 = p[J(1)];
  const T vm = nth == 1 ? v0 : p[J(nth - 1)];
  const T v2 = nth == 1 ? v1 : p[J(2)];
  p[J(0)] = v0;
  p[J(-1)] = vm;
  p[J(nth + 1)] = v1;
  p[J(nth + 2)] = v2;
}

// One thread per (column, array): Fc_r, Fc_th, Fc_z, p, lk_r, lk_th, lk_z.
__global__ void pcorr_wrap_kernel(PcorrArgs a) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const eaf_pcorr_fields_t& f = a.f;
  const long long ncol = (long long)(a.nr + 4) * (a.nz + 4);
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < 7 * ncol;
       w += (long long)gridDim.x * blockDim.x) {
    const int arr = (int)(w / ncol);
    const long long col = w % ncol;
    const long long base = (col % (a.nr + 4)) + a.sxy * (col / (a.nr + 4));
    switch (arr) {
      case 0: wrap_column(f.Fc_r, base, a.sx, a.nth); break;
      case 1: wrap_column(f.Fc_th, base, a.sx, a.nth); break;
      case 2: wrap_column(f.Fc_z, base, a.sx, a.nth); break;
      case 3: wrap_column(f.p, base, a.sx, a.nth); break;
      case 4: wrap_column(f.lk_r, base, a.sx, a.nth); break;
      case 5: wrap_column(f.lk_th, base, a.sx, a.nth); break;
      default: wrap_column(f.lk_z, base, a.sx, a.nth); break;
    }
  }
}

unsigned grid_for(long long work, int block) {
  long long g = (work + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (unsigned)g;
}

}  // namespace

cudaError_t launch_pcorr_f64(const eaf_pcorr_fields_t& f, int nr, int nth, int nz,
                             cudaStream_t st) {
  PcorrArgs a;
  a.f = f;
  a.nr = nr;
  a.nth = nth;
  a.nz = nz;
  a.sx = nr + 4;
  a.sxy = (long long)(nr + 4) * (nth + 4);
  a.nh = a.sxy * (nz + 4);
  const int block = 256;
  pcorr_update_kernel<<<grid_for(a.nh, block), block, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // The two dependent launches are programmatic: scheduled while the
  // previous grid drains, each waiting on it in griddepcontrol.wait.
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(block);
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(grid_for((long long)nr * nth * nz, block));
  e = cudaLaunchKernelEx(&cfg, pcorr_sealed_kernel, a);
  if (e != cudaSuccess) return e;
  cfg.gridDim = dim3(grid_for(7LL * (nr + 4) * (nz + 4), block));
  return cudaLaunchKernelEx(&cfg, pcorr_wrap_kernel, a);
}

}  // namespace eaf
