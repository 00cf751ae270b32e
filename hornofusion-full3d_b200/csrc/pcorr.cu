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

// correct_velocities (src/mod_pressure_3d.f90:711-742) at halo index q of
// interior cell (i, j, k) (1-based); the coordinate arrays start at -1.
__device__ __forceinline__ void correct_cell(const PcorrArgs& a, const eaf_phase_fields_t& ph,
                                             long long q, int i, int j, int k) {
  const double* pp = a.f.pp;
  const double al = ph.alpha[q], vo = a.f.vol[q];
  const bool skip_r = (i == 1) || (i == a.nr);
  if (!skip_r && fabs(ph.aP_ur[q]) > kSmallP) {
    const double dc = al * vo / ph.aP_ur[q];
    ph.ur[q] = ph.ur[q] - dc * (pp[q + 1] - pp[q - 1]) / (a.f.r[i + 2] - a.f.r[i]);
  }
  if (fabs(ph.aP_uth[q]) > kSmallP) {
    const double dc = al * vo / ph.aP_uth[q];
    ph.uth[q] = ph.uth[q] - dc * (pp[q + a.sx] - pp[q - a.sx]) /
                                (a.f.r[i + 1] * (a.f.theta[j + 2] - a.f.theta[j]));
  }
  const bool skip_z = (k == 1) || (k == a.nz);
  if (!skip_z && fabs(ph.aP_uz[q]) > kSmallP) {
    const double dc = al * vo / ph.aP_uz[q];
    ph.uz[q] = ph.uz[q] - dc * (pp[q + a.sxy] - pp[q - a.sxy]) / (a.f.z[k + 2] - a.f.z[k]);
  }
}

__global__ void pcorr_update_kernel(PcorrArgs a) {
  const eaf_pcorr_fields_t& f = a.f;
  const long long rows = a.nth + 4;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < a.nh;
       q += (long long)gridDim.x * blockDim.x) {
    // (:358-360) over the whole array
    const double pv = f.p[q] + f.alpha_p * f.pp[q];
    f.p[q] = fmax(-kHydroCap, fmin(kHydroCap, pv));
    const int i = (int)(q % a.sx) - 1;
    const long long t = q / a.sx;
    const int j = (int)(t % rows) - 1, k = (int)(t / rows) - 1;
    if (i < 1 || i > a.nr || j < 1 || j > a.nth || k < 1 || k > a.nz) continue;
    if (f.cell_type[q] == 0) continue;
    // (:333-345)
    const double* pp = f.pp;
    if (f.lk_r[q] == 1) f.Fc_r[q] = f.Fs_r[q] + f.ac_r[q] * (pp[q] - pp[q + 1]);
    if (f.lk_th[q] == 1) f.Fc_th[q] = f.Fs_th[q] + f.ac_th[q] * (pp[q] - pp[q + a.sx]);
    if (f.lk_z[q] == 1) f.Fc_z[q] = f.Fs_z[q] + f.ac_z[q] * (pp[q] - pp[q + a.sxy]);
    // (:354-356)
    if (f.act_l[q]) correct_cell(a, f.liq, q, i, j, k);
    if (f.has_gas && f.act_g[q]) correct_cell(a, f.gas, q, i, j, k);
  }
}

// (:373-395) with acc_nb (:451-458): neighbours in the order i-1, i+1,
// j-1, j+1, k-1, k+1, summed from 0.
__global__ void pcorr_sealed_kernel(PcorrArgs a) {
  const eaf_pcorr_fields_t& f = a.f;
  const long long n = (long long)a.nr * a.nth * a.nz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % a.nr) + 1;
    const long long t = c / a.nr;
    const int j = (int)(t % a.nth) + 1, k = (int)(t / a.nth) + 1;
    const long long q = (long long)(i + 1) + a.sx * (j + 1) + a.sxy * (k + 1);
    if (f.cell_type[q] == 0) continue;
    if (f.act_l[q] || f.act_g[q]) continue;
    const long long nb[6] = {q - 1, q + 1, q - a.sx, q + a.sx, q - a.sxy, q + a.sxy};
    double psum = 0.0;
    int nnb = 0;
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      const long long b = nb[u];
      if (f.cell_type[b] == 0) continue;
      if (!f.act_l[b] && !f.act_g[b]) continue;
      psum = psum + f.p[b];
      nnb = nnb + 1;
    }
    f.p[q] = nnb > 0 ? psum / (double)nnb : 0.0;
  }
}

// Serial theta-periodic copy (src/mod_mpi_topology.f90:303-311 and its int
// twin :686-692) of one (i, k) column of x, in statement order; with
// nth == 1 the second and fourth copies read what the first and third
// wrote, so they take the value from a register.
template <typename T>
__device__ __forceinline__ void wrap_column(T* x, long long col_base, long long sx, int nth) {
  T* p = x + col_base;
  auto J = [&](int j) { return (long long)(j + 1) * sx; };
  const T v0 = p[J(nth)];
  p[J(0)] = v0;
  p[J(-1)] = nth == 1 ? v0 : p[J(nth - 1)];
  const T v1 = p[J(1)];
  p[J(nth + 1)] = v1;
  p[J(nth + 2)] = nth == 1 ? v1 : p[J(2)];
}

__global__ void pcorr_wrap_kernel(PcorrArgs a) {
  const eaf_pcorr_fields_t& f = a.f;
  const long long ncol = (long long)(a.nr + 4) * (a.nz + 4);
  for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncol;
       col += (long long)gridDim.x * blockDim.x) {
    const long long base = (col % (a.nr + 4)) + a.sxy * (col / (a.nr + 4));
    wrap_column(f.Fc_r, base, a.sx, a.nth);
    wrap_column(f.Fc_th, base, a.sx, a.nth);
    wrap_column(f.Fc_z, base, a.sx, a.nth);
    wrap_column(f.lk_r, base, a.sx, a.nth);
    wrap_column(f.lk_th, base, a.sx, a.nth);
    wrap_column(f.lk_z, base, a.sx, a.nth);
    wrap_column(f.p, base, a.sx, a.nth);
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
  pcorr_sealed_kernel<<<grid_for((long long)nr * nth * nz, block), block, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  pcorr_wrap_kernel<<<grid_for((long long)(nr + 4) * (nz + 4), block), block, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace eaf
