// The C-ABI entries of the solvers around the CG on the same handle: the
// line-by-line TDMA and the transport residual, the post-CG corrections, the
// assembly of the pressure-correction equation and the whole pressure step.
// The handle and the CG's enqueue/finish steps come from handle.h.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "cg_kernels.h"
#include "eafcg.h"
#include "eafcg_internal.h"
#include "handle.h"

using eaf::HaloInputs;
using eaf::SolveResult;
using eaf::set_error;

namespace {

// ---------------------------------------------------------------------------
// Line-by-line TDMA sweeps and the transport residual on the handle's mesh.
// ---------------------------------------------------------------------------
int enqueue_tdma(eaf_cg* h, const HaloInputs& in, double* phi, int n_sweep) {
  if (!h->tdma_mbox) {
    EAF_CUDA(cudaMalloc((void**)&h->tdma_mbox,
                        sizeof(double) * eaf::tdma_mailbox_doubles(h->nr, h->nth, h->nz)));
  }
  if (!h->tdma_fac) {
    EAF_CUDA(cudaMalloc((void**)&h->tdma_fac,
                        sizeof(double) * eaf::tdma_factor_doubles(h->nr, h->nth, h->nz)));
  }
  h->last_grid = eaf::tdma_grid(h->nr, h->nth, h->nz);
  h->last_block = 64;
  h->last_cluster = 1;
  EAF_CUDA(cudaEventRecord(h->ev[1], h->st));
  EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
  if (n_sweep > 0) {
    EAF_CUDA(eaf::launch_tdma_f64(in, phi, h->nr, h->nth, h->nz, n_sweep, h->tdma_mbox,
                                  h->tdma_fac, h->ws, h->timeout_ns, h->st));
  }
  EAF_CUDA(cudaEventRecord(h->ev[3], h->st));
  EAF_CUDA(cudaEventRecord(h->ev[4], h->st));
  h->last_kernels = n_sweep > 0 ? 2 : 0;
  return EAF_OK;
}

int finish_tdma(eaf_cg* h, bool host_path, int n_sweep) {
  int err = 0;
  if (n_sweep > 0)
    EAF_CUDA(cudaMemcpyAsync(&h->res_h->status, h->ws.err, sizeof(int),
                             cudaMemcpyDeviceToHost, h->st));
  EAF_CUDA(cudaStreamSynchronize(h->st));
  if (n_sweep > 0) err = h->res_h->status;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[1], h->ev[4]) == cudaSuccess) h->last_solve_ms = ms;
  if (cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]) == cudaSuccess) h->last_kernel_ms = ms;
  if (host_path && cudaEventElapsedTime(&ms, h->ev[0], h->ev[5]) == cudaSuccess)
    h->last_e2e_ms = ms;
  return err;
}

int residual_launch_shape(const eaf_cg* h, int* grid, int* block) {
  const int b = 512;
  long long g = ((long long)h->d.n + 4095) / 4096;
  if (g < 1) g = 1;
  if (g > h->sms) g = h->sms;
  *grid = (int)g;
  *block = b;
  return EAF_OK;
}

int run_residual(eaf_cg* h, const HaloInputs& in, const double* phi, double* residual) {
  int grid, block;
  residual_launch_shape(h, &grid, &block);
  h->last_grid = grid;
  h->last_block = block;
  h->last_cluster = 1;
  EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
  EAF_CUDA(eaf::launch_residual_f64(in, phi, h->d, h->ws, h->timeout_ns, grid, block,
                                    h->st));
  EAF_CUDA(cudaEventRecord(h->ev[3], h->st));
  EAF_CUDA(cudaMemcpyAsync(h->res_h, h->ws.result, sizeof(SolveResult),
                           cudaMemcpyDeviceToHost, h->st));
  EAF_CUDA(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]) == cudaSuccess) h->last_kernel_ms = ms;
  h->last_kernels = 1;
  *residual = h->res_h->residual;
  return h->res_h->status;
}

// ---------------------------------------------------------------------------
// Post-CG corrections.
// ---------------------------------------------------------------------------
constexpr int kPcHalo = 26;  // halo double arrays of the mirror
constexpr int kPcInts = 6;

bool pcorr_fields_ok(const eaf_pcorr_fields_t* f) {
  if (!f) return false;
  const void* req[] = {f->pp,     f->Fs_r,   f->Fs_th,  f->Fs_z,      f->ac_r,
                       f->ac_th,  f->ac_z,   f->Fc_r,   f->Fc_th,     f->Fc_z,
                       f->vol,    f->r,      f->theta,  f->z,         f->p,
                       f->liq.alpha, f->liq.aP_ur, f->liq.aP_uth, f->liq.aP_uz,
                       f->liq.ur, f->liq.uth, f->liq.uz, f->lk_r,    f->lk_th,
                       f->lk_z,   f->cell_type, f->act_l, f->act_g};
  for (const void* q : req)
    if (!q) return false;
  if (f->has_gas) {
    const void* gas[] = {f->gas.alpha, f->gas.aP_ur, f->gas.aP_uth, f->gas.aP_uz,
                         f->gas.ur,    f->gas.uth,   f->gas.uz};
    for (const void* q : gas)
      if (!q) return false;
  }
  return true;
}

int run_pcorr(eaf_cg* h, const eaf_pcorr_fields_t& f) {
  EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
  EAF_CUDA(eaf::launch_pcorr_f64(f, h->nr, h->nth, h->nz, h->st));
  EAF_CUDA(cudaEventRecord(h->ev[3], h->st));
  h->last_kernels = 3;
  return EAF_OK;
}

// ---------------------------------------------------------------------------
// Pressure-equation assembly.
// ---------------------------------------------------------------------------
constexpr int kAsmIn = 24;   // halo double inputs of the mirror
constexpr int kAsmOut = 18;  // halo double outputs
constexpr int kAsmInts = 7;

bool assembly_fields_ok(const eaf_assembly_fields_t* f) {
  if (!f || !(f->dt > 0.0)) return false;
  const void* req[] = {f->cell_type, f->outlet, f->act_l, f->act_g, f->vol, f->Ar, f->Ath,
                       f->Az, f->r, f->theta, f->z, f->p,
                       f->liq.alpha, f->liq.rho, f->liq.ur, f->liq.uth, f->liq.uz,
                       f->liq.aP_ur, f->liq.aP_uth, f->liq.aP_uz,
                       f->aW, f->aE, f->aS, f->aN, f->aB, f->aT, f->aP, f->Su, f->pp,
                       f->Fs_r, f->Fs_th, f->Fs_z, f->ac_r, f->ac_th, f->ac_z,
                       f->Fc_r, f->Fc_th, f->Fc_z, f->lk_r, f->lk_th, f->lk_z};
  for (const void* q : req)
    if (!q) return false;
  if (f->liq_room_valid && !f->liq_room) return false;
  if (f->gas_in_poisson) {
    const void* gas[] = {f->liq_T, f->gas.alpha, f->gas.rho, f->gas.ur, f->gas.uth,
                         f->gas.uz, f->gas.aP_ur, f->gas.aP_uth, f->gas.aP_uz};
    for (const void* q : gas)
      if (!q) return false;
  }
  if (f->gas_compressibility && (!f->gas.alpha || !f->gas.rho || !f->gas_T_old)) return false;
  return true;
}

// Fields the kernels never read are cleared, so a flag that is off cannot
// lead them to a stale pointer.
eaf_assembly_fields_t assembly_normalised(const eaf_assembly_fields_t& f) {
  eaf_assembly_fields_t d = f;
  d.liq_room_valid = f.liq_room_valid ? 1 : 0;
  d.gas_in_poisson = f.gas_in_poisson ? 1 : 0;
  d.gas_compressibility = f.gas_compressibility ? 1 : 0;
  if (!d.liq_room_valid) d.liq_room = nullptr;
  if (!d.gas_in_poisson) {
    d.liq_T = nullptr;
    d.gas.ur = d.gas.uth = d.gas.uz = nullptr;
    d.gas.aP_ur = d.gas.aP_uth = d.gas.aP_uz = nullptr;
    if (!d.gas_compressibility) d.gas.alpha = d.gas.rho = nullptr;
  }
  if (!d.gas_compressibility) d.gas_T_old = nullptr;
  return d;
}

int run_assemble(eaf_cg* h, const eaf_assembly_fields_t& f) {
  if (!h->asm_s) {
    EAF_CUDA(cudaMalloc((void**)&h->asm_s,
                        sizeof(double) * eaf::assembly_scratch_doubles(h->nr, h->nth, h->nz)));
  }
  EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
  EAF_CUDA(eaf::launch_assemble_f64(f, h->nr, h->nth, h->nz, h->asm_s, h->st));
  EAF_CUDA(cudaEventRecord(h->ev[3], h->st));
  EAF_CUDA(cudaMemcpyAsync(&h->res_h->residual,
                           eaf::assembly_result(h->asm_s, h->nr, h->nth, h->nz),
                           sizeof(double), cudaMemcpyDeviceToHost, h->st));
  h->last_kernels = 4;
  return EAF_OK;
}

// Uploads the inputs the switches read into the handle's assembly mirror
// (allocated on first use) and points d at the mirror: mirror slots 0 vol,
// 1-3 Ar Ath Az, 4 p, 5 liq_room, 6-13 liquid state, 14 liq_T, 15-22 gas
// state, 23 gas_T_old, 24-41 outputs (aW .. Fc_z), then the coordinates;
// ints: cell_type, outlet, act_l, act_g, lk_r, lk_th, lk_z.
int stage_assembly(eaf_cg* h, const eaf_assembly_fields_t& src, eaf_assembly_fields_t& d) {
  const size_t nh = h->nh;
  const size_t nc = (size_t)(h->nr + 4) + (h->nth + 4) + (h->nz + 4);
  if (!h->asm_d) {
    EAF_CUDA(cudaMalloc((void**)&h->asm_d, sizeof(double) * ((kAsmIn + kAsmOut) * nh + nc)));
  }
  if (!h->asm_i) {
    EAF_CUDA(cudaMalloc((void**)&h->asm_i, sizeof(int) * kAsmInts * nh));
  }
  d = src;
  auto slot = [&](int i) { return h->asm_d + (size_t)i * nh; };
  const double* in[kAsmIn] = {src.vol, src.Ar, src.Ath, src.Az, src.p, src.liq_room,
                              src.liq.alpha, src.liq.rho, src.liq.ur, src.liq.uth,
                              src.liq.uz, src.liq.aP_ur, src.liq.aP_uth, src.liq.aP_uz,
                              src.liq_T,
                              src.gas.alpha, src.gas.rho, src.gas.ur, src.gas.uth,
                              src.gas.uz, src.gas.aP_ur, src.gas.aP_uth, src.gas.aP_uz,
                              src.gas_T_old};
  const double** din[kAsmIn] = {&d.vol, &d.Ar, &d.Ath, &d.Az, &d.p, &d.liq_room,
                                &d.liq.alpha, &d.liq.rho, &d.liq.ur, &d.liq.uth,
                                &d.liq.uz, &d.liq.aP_ur, &d.liq.aP_uth, &d.liq.aP_uz,
                                &d.liq_T,
                                &d.gas.alpha, &d.gas.rho, &d.gas.ur, &d.gas.uth,
                                &d.gas.uz, &d.gas.aP_ur, &d.gas.aP_uth, &d.gas.aP_uz,
                                &d.gas_T_old};
  for (int i = 0; i < kAsmIn; ++i) {
    if (!in[i]) continue;  // not read under these switches
    EAF_CUDA(cudaMemcpyAsync(slot(i), in[i], nh * sizeof(double), cudaMemcpyHostToDevice,
                             h->st));
    *din[i] = slot(i);
  }
  double* coords = slot(kAsmIn + kAsmOut);
  EAF_CUDA(cudaMemcpyAsync(coords, src.r, (h->nr + 4) * sizeof(double),
                           cudaMemcpyHostToDevice, h->st));
  EAF_CUDA(cudaMemcpyAsync(coords + h->nr + 4, src.theta, (h->nth + 4) * sizeof(double),
                           cudaMemcpyHostToDevice, h->st));
  EAF_CUDA(cudaMemcpyAsync(coords + h->nr + 4 + h->nth + 4, src.z,
                           (h->nz + 4) * sizeof(double), cudaMemcpyHostToDevice, h->st));
  d.r = coords;
  d.theta = coords + h->nr + 4;
  d.z = coords + h->nr + 4 + h->nth + 4;
  const int* in_i[4] = {src.cell_type, src.outlet, src.act_l, src.act_g};
  const int** din_i[4] = {&d.cell_type, &d.outlet, &d.act_l, &d.act_g};
  for (int i = 0; i < 4; ++i) {
    EAF_CUDA(cudaMemcpyAsync(h->asm_i + (size_t)i * nh, in_i[i], nh * sizeof(int),
                             cudaMemcpyHostToDevice, h->st));
    *din_i[i] = h->asm_i + (size_t)i * nh;
  }
  double** dout[kAsmOut] = {&d.aW, &d.aE, &d.aS, &d.aN, &d.aB, &d.aT, &d.aP, &d.Su, &d.pp,
                            &d.Fs_r, &d.Fs_th, &d.Fs_z, &d.ac_r, &d.ac_th, &d.ac_z,
                            &d.Fc_r, &d.Fc_th, &d.Fc_z};
  for (int i = 0; i < kAsmOut; ++i) *dout[i] = slot(kAsmIn + i);
  d.lk_r = h->asm_i + 4 * nh;
  d.lk_th = h->asm_i + 5 * nh;
  d.lk_z = h->asm_i + 6 * nh;
  return EAF_OK;
}

// Downloads the assembly's outputs from the mirror; with `step`, also the
// arrays the post-CG corrections update (p and the velocities of the phases
// in the equation).
int fetch_assembly(eaf_cg* h, const eaf_assembly_fields_t& src, const eaf_assembly_fields_t& d,
                   bool step) {
  const size_t bytes = h->nh * sizeof(double);
  double* out_h[kAsmOut] = {src.aW, src.aE, src.aS, src.aN, src.aB, src.aT, src.aP,
                            src.Su, src.pp, src.Fs_r, src.Fs_th, src.Fs_z,
                            src.ac_r, src.ac_th, src.ac_z, src.Fc_r, src.Fc_th, src.Fc_z};
  const double* out_d[kAsmOut] = {d.aW, d.aE, d.aS, d.aN, d.aB, d.aT, d.aP, d.Su, d.pp,
                                  d.Fs_r, d.Fs_th, d.Fs_z, d.ac_r, d.ac_th, d.ac_z,
                                  d.Fc_r, d.Fc_th, d.Fc_z};
  for (int i = 0; i < kAsmOut; ++i)
    EAF_CUDA(cudaMemcpyAsync(out_h[i], out_d[i], bytes, cudaMemcpyDeviceToHost, h->st));
  int* lk_h[3] = {src.lk_r, src.lk_th, src.lk_z};
  const int* lk_d[3] = {d.lk_r, d.lk_th, d.lk_z};
  for (int i = 0; i < 3; ++i)
    EAF_CUDA(cudaMemcpyAsync(lk_h[i], lk_d[i], h->nh * sizeof(int), cudaMemcpyDeviceToHost,
                             h->st));
  if (step) {
    const double* upd_d[7] = {d.p, d.liq.ur, d.liq.uth, d.liq.uz, d.gas.ur, d.gas.uth,
                              d.gas.uz};
    const double* upd_h[7] = {src.p, src.liq.ur, src.liq.uth, src.liq.uz, src.gas.ur,
                              src.gas.uth, src.gas.uz};
    const int n = d.gas_in_poisson ? 7 : 4;
    for (int i = 0; i < n; ++i)
      EAF_CUDA(cudaMemcpyAsync(const_cast<double*>(upd_h[i]), upd_d[i], bytes,
                               cudaMemcpyDeviceToHost, h->st));
  }
  return EAF_OK;
}

// The serial numerics of solve_pressure_correction (src/mod_pressure_3d.f90:
// 135-397) on device arrays, back to back on the handle's stream: the
// assembly (launch_assemble_f64), the CG on its coefficients into pp
// (cg_3d_mpi, :316-318), then the post-CG corrections (launch_pcorr_f64)
// over the same arrays -- p and the velocities are updated in place. As the
// reference (:320), the corrections run whatever the CG returned, and a NaN
// CG residual replaces the continuity residual.
int run_step(eaf_cg* h, const eaf_assembly_fields_t& d, double alpha_p, int max_iter,
             double tol, double* residual, double* cg_res, int* n_iter) {
  if (!h->asm_s) {
    EAF_CUDA(cudaMalloc((void**)&h->asm_s,
                        sizeof(double) * eaf::assembly_scratch_doubles(h->nr, h->nth, h->nz)));
  }
  for (int i = 0; i < 2; ++i)
    if (!h->step_ev[i]) EAF_CUDA(cudaEventCreate(&h->step_ev[i]));
  EAF_CUDA(cudaEventRecord(h->step_ev[0], h->st));
  EAF_CUDA(eaf::launch_assemble_f64(d, h->nr, h->nth, h->nz, h->asm_s, h->st));
  HaloInputs in = {d.aW, d.aE, d.aS, d.aN, d.aB, d.aT, d.aP, d.Su, d.pp};
  SolveOpts o = {false, max_iter, 0, tol, 0.0};
  int rc = enqueue_solve(h, in, d.pp, o);
  if (rc != EAF_OK) return rc;
  const int cg_kernels = h->last_kernels;
  auto mut = [](const double* p) { return const_cast<double*>(p); };
  eaf_pcorr_fields_t pc = {};
  pc.pp = d.pp;
  pc.Fs_r = d.Fs_r; pc.Fs_th = d.Fs_th; pc.Fs_z = d.Fs_z;
  pc.ac_r = d.ac_r; pc.ac_th = d.ac_th; pc.ac_z = d.ac_z;
  pc.Fc_r = d.Fc_r; pc.Fc_th = d.Fc_th; pc.Fc_z = d.Fc_z;
  pc.vol = d.vol;
  pc.r = d.r; pc.theta = d.theta; pc.z = d.z;
  pc.p = mut(d.p);
  pc.liq = eaf_phase_fields_t{d.liq.alpha, d.liq.aP_ur, d.liq.aP_uth, d.liq.aP_uz,
                              mut(d.liq.ur), mut(d.liq.uth), mut(d.liq.uz)};
  if (d.gas_in_poisson)
    pc.gas = eaf_phase_fields_t{d.gas.alpha, d.gas.aP_ur, d.gas.aP_uth, d.gas.aP_uz,
                                mut(d.gas.ur), mut(d.gas.uth), mut(d.gas.uz)};
  pc.lk_r = d.lk_r; pc.lk_th = d.lk_th; pc.lk_z = d.lk_z;
  pc.cell_type = d.cell_type;
  pc.act_l = d.act_l;
  pc.act_g = d.act_g;
  pc.has_gas = d.gas_in_poisson;
  pc.alpha_p = alpha_p;
  EAF_CUDA(eaf::launch_pcorr_f64(pc, h->nr, h->nth, h->nz, h->st));
  EAF_CUDA(cudaEventRecord(h->step_ev[1], h->st));
  const int st = finish_solve(h, false, cg_res, n_iter, nullptr);  // synchronises
  if (st != EAF_OK && st != EAF_ENONFINITE) return st;
  double cont = 0.0;
  EAF_CUDA(cudaMemcpy(&cont, eaf::assembly_result(h->asm_s, h->nr, h->nth, h->nz),
                      sizeof(double), cudaMemcpyDeviceToHost));
  *residual = *cg_res != *cg_res ? *cg_res : cont;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->step_ev[0], h->step_ev[1]) == cudaSuccess)
    h->last_kernel_ms = ms;
  h->last_kernels = 4 + cg_kernels + 3;
  return st;
}

}  // namespace

extern "C" {

int eaf_tdma_3d_f64(eaf_cg_t h, const double* aW, const double* aE, const double* aS,
                    const double* aN, const double* aB, const double* aT,
                    const double* aP, const double* Su, double* phi, int n_sweep) {
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  if (!h || !phi || any_null(arr, 8)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  const size_t bytes = h->nh * sizeof(double);
  EAF_CUDA(cudaEventRecord(h->ev[0], h->st));
  for (int i = 0; i < 8; ++i)
    EAF_CUDA(cudaMemcpyAsync(h->stage[i], arr[i], bytes, cudaMemcpyHostToDevice, h->st));
  EAF_CUDA(cudaMemcpyAsync(h->stage[8], phi, bytes, cudaMemcpyHostToDevice, h->st));
  HaloInputs in = {h->stage[0], h->stage[1], h->stage[2], h->stage[3], h->stage[4],
                   h->stage[5], h->stage[6], h->stage[7], h->stage[8]};
  int rc = enqueue_tdma(h, in, h->stage[8], n_sweep);
  if (rc != EAF_OK) return rc;
  EAF_CUDA(cudaMemcpyAsync(phi, h->stage[8], bytes, cudaMemcpyDeviceToHost, h->st));
  EAF_CUDA(cudaEventRecord(h->ev[5], h->st));
  return finish_tdma(h, true, n_sweep);
}

int eaf_tdma_3d_f64_device(eaf_cg_t h, const double* aW, const double* aE,
                           const double* aS, const double* aN, const double* aB,
                           const double* aT, const double* aP, const double* Su,
                           double* phi, int n_sweep) {
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  if (!h || !phi || any_null(arr, 8)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  HaloInputs in = {arr[0], arr[1], arr[2], arr[3], arr[4], arr[5], arr[6], arr[7], phi};
  int rc = enqueue_tdma(h, in, phi, n_sweep);
  if (rc != EAF_OK) return rc;
  return finish_tdma(h, false, n_sweep);
}

int eaf_residual_3d_f64(eaf_cg_t h, const double* aW, const double* aE, const double* aS,
                        const double* aN, const double* aB, const double* aT,
                        const double* aP, const double* Su, const double* phi,
                        double* residual) {
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  if (!h || !phi || !residual || any_null(arr, 8)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  const size_t bytes = h->nh * sizeof(double);
  for (int i = 0; i < 8; ++i)
    EAF_CUDA(cudaMemcpyAsync(h->stage[i], arr[i], bytes, cudaMemcpyHostToDevice, h->st));
  EAF_CUDA(cudaMemcpyAsync(h->stage[8], phi, bytes, cudaMemcpyHostToDevice, h->st));
  HaloInputs in = {h->stage[0], h->stage[1], h->stage[2], h->stage[3], h->stage[4],
                   h->stage[5], h->stage[6], h->stage[7], h->stage[8]};
  return run_residual(h, in, h->stage[8], residual);
}

int eaf_residual_3d_f64_device(eaf_cg_t h, const double* aW, const double* aE,
                               const double* aS, const double* aN, const double* aB,
                               const double* aT, const double* aP, const double* Su,
                               const double* phi, double* residual) {
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  if (!h || !phi || !residual || any_null(arr, 8)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  HaloInputs in = {arr[0], arr[1], arr[2], arr[3], arr[4], arr[5], arr[6], arr[7], phi};
  return run_residual(h, in, phi, residual);
}

int eaf_pressure_correct_f64_device(eaf_cg_t h, const eaf_pcorr_fields_t* f) {
  if (!h || !pcorr_fields_ok(f)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  eaf_pcorr_fields_t d = *f;
  if (!d.has_gas) d.gas = eaf_phase_fields_t{};
  int rc = run_pcorr(h, d);
  if (rc != EAF_OK) return rc;
  EAF_CUDA(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]) == cudaSuccess) h->last_kernel_ms = ms;
  return EAF_OK;
}

int eaf_pressure_correct_f64(eaf_cg_t h, const eaf_pcorr_fields_t* f) {
  if (!h || !pcorr_fields_ok(f)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  const size_t nh = h->nh;
  const size_t nc = (size_t)(h->nr + 4) + (h->nth + 4) + (h->nz + 4);
  if (!h->pc_d) {
    EAF_CUDA(cudaMalloc((void**)&h->pc_d, sizeof(double) * (kPcHalo * nh + nc)));
  }
  if (!h->pc_i) {
    EAF_CUDA(cudaMalloc((void**)&h->pc_i, sizeof(int) * kPcInts * nh));
  }
  double* D = h->pc_d;
  int* I = h->pc_i;
  eaf_pcorr_fields_t d = *f;
  // mirror slots: 0 pp, 1-3 Fs, 4-6 ac, 7-9 Fc, 10 vol, 11 p, 12-18 liq, 19-25 gas
  const double* src_in[] = {f->pp, f->Fs_r, f->Fs_th, f->Fs_z, f->ac_r, f->ac_th,
                            f->ac_z, f->Fc_r, f->Fc_th, f->Fc_z, f->vol, f->p,
                            f->liq.alpha, f->liq.aP_ur, f->liq.aP_uth, f->liq.aP_uz,
                            f->liq.ur, f->liq.uth, f->liq.uz,
                            f->gas.alpha, f->gas.aP_ur, f->gas.aP_uth, f->gas.aP_uz,
                            f->gas.ur, f->gas.uth, f->gas.uz};
  const int n_in = f->has_gas ? 26 : 19;
  EAF_CUDA(cudaEventRecord(h->ev[0], h->st));
  for (int i = 0; i < n_in; ++i)
    EAF_CUDA(cudaMemcpyAsync(D + (size_t)i * nh, src_in[i], nh * sizeof(double),
                             cudaMemcpyHostToDevice, h->st));
  double* coords = D + (size_t)kPcHalo * nh;
  EAF_CUDA(cudaMemcpyAsync(coords, f->r, (h->nr + 4) * sizeof(double),
                           cudaMemcpyHostToDevice, h->st));
  EAF_CUDA(cudaMemcpyAsync(coords + h->nr + 4, f->theta, (h->nth + 4) * sizeof(double),
                           cudaMemcpyHostToDevice, h->st));
  EAF_CUDA(cudaMemcpyAsync(coords + h->nr + 4 + h->nth + 4, f->z,
                           (h->nz + 4) * sizeof(double), cudaMemcpyHostToDevice, h->st));
  const int* src_i[] = {f->lk_r, f->lk_th, f->lk_z, f->cell_type, f->act_l, f->act_g};
  for (int i = 0; i < kPcInts; ++i)
    EAF_CUDA(cudaMemcpyAsync(I + (size_t)i * nh, src_i[i], nh * sizeof(int),
                             cudaMemcpyHostToDevice, h->st));
  auto slot = [&](int i) { return D + (size_t)i * nh; };
  d.pp = slot(0);
  d.Fs_r = slot(1); d.Fs_th = slot(2); d.Fs_z = slot(3);
  d.ac_r = slot(4); d.ac_th = slot(5); d.ac_z = slot(6);
  d.Fc_r = slot(7); d.Fc_th = slot(8); d.Fc_z = slot(9);
  d.vol = slot(10); d.p = slot(11);
  d.liq = eaf_phase_fields_t{slot(12), slot(13), slot(14), slot(15), slot(16), slot(17),
                             slot(18)};
  d.gas = f->has_gas ? eaf_phase_fields_t{slot(19), slot(20), slot(21), slot(22), slot(23),
                                          slot(24), slot(25)}
                     : eaf_phase_fields_t{};
  d.r = coords;
  d.theta = coords + h->nr + 4;
  d.z = coords + h->nr + 4 + h->nth + 4;
  d.lk_r = I; d.lk_th = I + nh; d.lk_z = I + 2 * nh;
  d.cell_type = I + 3 * nh; d.act_l = I + 4 * nh; d.act_g = I + 5 * nh;
  int rc = run_pcorr(h, d);
  if (rc != EAF_OK) return rc;
  double* dst_out[] = {f->Fc_r, f->Fc_th, f->Fc_z, f->p, f->liq.ur, f->liq.uth, f->liq.uz,
                       f->gas.ur, f->gas.uth, f->gas.uz};
  const int slots_out[] = {7, 8, 9, 11, 16, 17, 18, 23, 24, 25};
  const int n_out = f->has_gas ? 10 : 7;
  for (int i = 0; i < n_out; ++i)
    EAF_CUDA(cudaMemcpyAsync(dst_out[i], slot(slots_out[i]), nh * sizeof(double),
                             cudaMemcpyDeviceToHost, h->st));
  int* lk_out[] = {f->lk_r, f->lk_th, f->lk_z};
  for (int i = 0; i < 3; ++i)
    EAF_CUDA(cudaMemcpyAsync(lk_out[i], I + (size_t)i * nh, nh * sizeof(int),
                             cudaMemcpyDeviceToHost, h->st));
  EAF_CUDA(cudaEventRecord(h->ev[5], h->st));
  EAF_CUDA(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]) == cudaSuccess) h->last_kernel_ms = ms;
  if (cudaEventElapsedTime(&ms, h->ev[0], h->ev[5]) == cudaSuccess) h->last_e2e_ms = ms;
  return EAF_OK;
}

int eaf_pressure_assemble_f64_device(eaf_cg_t h, const eaf_assembly_fields_t* f,
                                     double* residual) {
  if (!h || !residual || !assembly_fields_ok(f)) return EAF_EINVAL;
  if (h->nh > (size_t)INT32_MAX) return EAF_EUNSUPPORTED;  // 32-bit element indices
  eaf::DeviceGuard guard(h->device);
  const eaf_assembly_fields_t d = assembly_normalised(*f);
  int rc = run_assemble(h, d);
  if (rc != EAF_OK) return rc;
  EAF_CUDA(cudaStreamSynchronize(h->st));
  *residual = h->res_h->residual;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]) == cudaSuccess) h->last_kernel_ms = ms;
  return EAF_OK;
}

int eaf_pressure_assemble_f64(eaf_cg_t h, const eaf_assembly_fields_t* f, double* residual) {
  if (!h || !residual || !assembly_fields_ok(f)) return EAF_EINVAL;
  if (h->nh > (size_t)INT32_MAX) return EAF_EUNSUPPORTED;  // 32-bit element indices
  eaf::DeviceGuard guard(h->device);
  const eaf_assembly_fields_t src = assembly_normalised(*f);
  eaf_assembly_fields_t d;
  EAF_CUDA(cudaEventRecord(h->ev[0], h->st));
  int rc = stage_assembly(h, src, d);
  if (rc == EAF_OK) rc = run_assemble(h, d);
  if (rc == EAF_OK) rc = fetch_assembly(h, src, d, false);
  if (rc != EAF_OK) return rc;
  EAF_CUDA(cudaEventRecord(h->ev[5], h->st));
  EAF_CUDA(cudaStreamSynchronize(h->st));
  *residual = h->res_h->residual;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]) == cudaSuccess) h->last_kernel_ms = ms;
  if (cudaEventElapsedTime(&ms, h->ev[0], h->ev[5]) == cudaSuccess) h->last_e2e_ms = ms;
  return EAF_OK;
}

int eaf_pressure_step_f64_device(eaf_cg_t h, const eaf_assembly_fields_t* f, double alpha_p,
                                 int max_iter, double tol, double* residual, double* cg_res,
                                 int* n_iter) {
  if (!h || !residual || !cg_res || !n_iter || !assembly_fields_ok(f)) return EAF_EINVAL;
  if (h->nh > (size_t)INT32_MAX) return EAF_EUNSUPPORTED;
  eaf::DeviceGuard guard(h->device);
  return run_step(h, assembly_normalised(*f), alpha_p, max_iter, tol, residual, cg_res,
                  n_iter);
}

int eaf_pressure_step_f64(eaf_cg_t h, const eaf_assembly_fields_t* f, double alpha_p,
                          int max_iter, double tol, double* residual, double* cg_res,
                          int* n_iter) {
  if (!h || !residual || !cg_res || !n_iter || !assembly_fields_ok(f)) return EAF_EINVAL;
  if (h->nh > (size_t)INT32_MAX) return EAF_EUNSUPPORTED;
  eaf::DeviceGuard guard(h->device);
  const eaf_assembly_fields_t src = assembly_normalised(*f);
  eaf_assembly_fields_t d;
  EAF_CUDA(cudaEventRecord(h->ev[0], h->st));
  int rc = stage_assembly(h, src, d);
  if (rc != EAF_OK) return rc;
  const int st = run_step(h, d, alpha_p, max_iter, tol, residual, cg_res, n_iter);
  if (st != EAF_OK && st != EAF_ENONFINITE) return st;
  rc = fetch_assembly(h, src, d, true);
  if (rc != EAF_OK) return rc;
  EAF_CUDA(cudaEventRecord(h->ev[5], h->st));
  EAF_CUDA(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[0], h->ev[5]) == cudaSuccess) h->last_e2e_ms = ms;
  return st;
}

}  // extern "C"
