// C-ABI shim of libeafcg.so: handle lifetime, device buffers, uploads,
// launches, result readback and timing for the single-system solvers.
// The public contract is documented in include/eafcg.h.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <new>

#include "cg_kernels.h"
#include "eafcg.h"
#include "eafcg_internal.h"
#include "tune_table.h"

using eaf::GroupWs;
using eaf::HaloInputs;
using eaf::MeshDims;
using eaf::SolveResult;
using eaf::SysF32;
using eaf::SysF64;

namespace {

constexpr int kPartSlots = 8;
constexpr int kDefaultBlock = 512;
constexpr uint64_t kDefaultTimeoutNs = 2000ull * 1000ull * 1000ull;

}  // namespace

struct eaf_cg {
  int nr, nth, nz, device;
  MeshDims d;
  size_t nh;  // halo-layout elements per array
  cudaStream_t st;
  double* stage[9];  // aW aE aS aN aB aT aP Su phi, halo layout (host path)
  SysF64 s;
  SysF32 f;
  bool have_f32;
  GroupWs ws;
  SolveResult* res_h;  // pinned
  int block, grid;     // 0 = automatic
  int sms;
  uint64_t timeout_ns;
  cudaEvent_t ev[6];   // e2e0, solve0, kern0, kern1, solve1, e2e1
  double last_solve_ms, last_kernel_ms, last_e2e_ms;
  int last_sym, last_kernels;
  int last_grid, last_block;
  double* tdma_mbox;  // TDMA line hand-over slots (lazy)
  double* tdma_fac;  // TDMA line factors (lazy)
  double* pc_d;      // post-CG correction mirror: doubles (lazy)
  int* pc_i;         // post-CG correction mirror: ints (lazy)
  int form;          // EAF_CG_FORM_*: the FP64 solver's recurrences
  double* asm_d;     // assembly mirror: doubles (lazy)
  int* asm_i;        // assembly mirror: ints (lazy)
  double* asm_s;     // assembly scratch: gradients, partials, residual (lazy)
  cudaEvent_t step_ev[2];  // span of a whole pressure step (lazy)
};

namespace eaf {

thread_local char g_last_error[256];

void set_error(const char* what, cudaError_t e) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what,
           e == cudaSuccess ? "ok" : cudaGetErrorString(e));
}

void set_error_text(const char* msg) {
  snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

DeviceGuard::DeviceGuard(int dev) : prev_(-1), ok_(false) {
  if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
  ok_ = cudaSetDevice(dev) == cudaSuccess;
}
DeviceGuard::~DeviceGuard() {
  if (prev_ >= 0) cudaSetDevice(prev_);
}

}  // namespace eaf

using eaf::set_error;

#define EAF_CUDA(call)                     \
  do {                                     \
    cudaError_t e_ = (call);               \
    if (e_ != cudaSuccess) {               \
      set_error(#call, e_);                \
      return EAF_ECUDA;                    \
    }                                      \
  } while (0)

static void free_handle(eaf_cg* h) {
  for (int i = 0; i < 9; ++i) cudaFree(h->stage[i]);
  double* f64[] = {h->s.aP, h->s.aE, h->s.aN, h->s.aT, h->s.aW, h->s.aS, h->s.aB,
                   h->s.b,  h->s.x,  h->s.r,  h->s.p,  h->s.q,  h->s.p2, h->s.z,
                   h->s.s0, h->s.s1, h->s.dinv};
  for (double* p : f64) cudaFree(p);
  cudaFree(h->s.asym);
  float* f32[] = {h->f.aP, h->f.aE, h->f.aN, h->f.aT, h->f.aW, h->f.aS, h->f.aB,
                  h->f.r,  h->f.z,  h->f.q,  h->f.e,  h->f.p,  h->f.p2};
  for (float* p : f32) cudaFree(p);
  cudaFree(h->ws.part);
  cudaFree(h->ws.counter);
  cudaFree(h->ws.err);
  cudaFree(h->ws.result);
  cudaFree(h->tdma_mbox);
  cudaFree(h->tdma_fac);
  cudaFree(h->pc_d);
  cudaFree(h->pc_i);
  cudaFree(h->asm_d);
  cudaFree(h->asm_i);
  cudaFree(h->asm_s);
  for (int i = 0; i < 2; ++i)
    if (h->step_ev[i]) cudaEventDestroy(h->step_ev[i]);
  if (h->res_h) cudaFreeHost(h->res_h);
  for (int i = 0; i < 6; ++i)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  if (h->st) cudaStreamDestroy(h->st);
}

static int max_coresident(const void* kernel, int block, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) !=
      cudaSuccess)
    return 0;
  return per_sm * sms;
}

// Launch shape for a persistent kernel over n cells: an explicit
// eaf_cg_set_launch shape, else the tuned shape of this mesh (FP64 solver),
// else one 1024-thread block up to 8192 cells or one 512-thread block per
// 2048 cells; capped by co-residency of the kernel (variant) that runs
// blocks of that size.
static void pick_launch(const eaf_cg* h, bool f64, int* grid, int* block) {
  auto kernel_for = [f64, h](int b) {
    if (!f64) return eaf::cg_mixed_kernel_ptr();
    return h->form == EAF_CG_FORM_ONE_REDUCTION ? eaf::cg1_f64_kernel_ptr(b)
                                                : eaf::cg_f64_kernel_ptr(b, h->d.n);
  };
  int b = h->block > 0 ? h->block : kDefaultBlock;
  int g;
  int tb = 0, tg = 0;
  if (h->block == 0 && h->grid == 0 && f64 &&
      eaf::tuned_single_launch(h->nr, h->nth, h->nz, &tb, &tg)) {
    b = tb;
    g = tg;
  } else if (h->grid > 0) {
    g = h->grid;
  } else if (h->d.n <= 8192) {
    b = h->block > 0 ? h->block : 1024;
    g = 1;
  } else {
    long long want = ((long long)h->d.n + (long long)b * 4 - 1) / ((long long)b * 4);
    g = (int)(want < 1 ? 1 : want);
  }
  const int cap = max_coresident(kernel_for(b), b, h->sms);
  if (cap > 0 && g > cap) g = cap;
  if (g > h->sms * 8) g = h->sms * 8;
  *grid = g;
  *block = b;
}

extern "C" {

const char* eaf_status_string(int s) {
  switch (s) {
    case EAF_OK: return "EAF_OK";
    case EAF_ECUDA: return "EAF_ECUDA";
    case EAF_EINVAL: return "EAF_EINVAL";
    case EAF_ENONFINITE: return "EAF_ENONFINITE";
    case EAF_ETIMEOUT: return "EAF_ETIMEOUT";
    case EAF_EUNSUPPORTED: return "EAF_EUNSUPPORTED";
    case EAF_ENOMEM: return "EAF_ENOMEM";
    case EAF_EADMIT: return "EAF_EADMIT";
    case EAF_EBUSY: return "EAF_EBUSY";
    case EAF_ECLOSED: return "EAF_ECLOSED";
    default: return "EAF_UNKNOWN";
  }
}

const char* eaf_last_error(void) { return eaf::g_last_error; }

const char* eaf_version(void) { return "eafcg-b200 0.1 (sm_100a)"; }

int eaf_cg_create_mesh(eaf_cg_t* out, int nr, int nth, int nz, int is_parallel,
                       int device) {
  if (!out) return EAF_EINVAL;
  *out = nullptr;
  if (is_parallel) return EAF_EUNSUPPORTED;
  if (nr < 1 || nth < 1 || nz < 1) return EAF_EINVAL;
  const long long n = (long long)nr * nth * nz;
  const long long nh = (long long)(nr + 4) * (nth + 4) * (nz + 4);
  if (nh >= (1ll << 31)) return EAF_EINVAL;
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) {
    set_error("cudaSetDevice", cudaErrorInvalidDevice);
    return EAF_ECUDA;
  }
  eaf_cg* h = new (std::nothrow) eaf_cg;
  if (!h) return EAF_ENOMEM;
  memset(h, 0, sizeof(*h));
  h->nr = nr;
  h->nth = nth;
  h->nz = nz;
  h->device = device;
  h->d = eaf::make_dims(nr, nth, nz);
  h->nh = (size_t)nh;
  h->timeout_ns = kDefaultTimeoutNs;
  int rc = EAF_OK;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
  for (int i = 0; i < 9; ++i) alloc((void**)&h->stage[i], h->nh * sizeof(double));
  double** f64[] = {&h->s.aP, &h->s.aE, &h->s.aN, &h->s.aT, &h->s.aW,
                    &h->s.aS, &h->s.aB, &h->s.b,  &h->s.x,  &h->s.r,
                    &h->s.p,  &h->s.q,  &h->s.p2, &h->s.z, &h->s.s0, &h->s.s1,
                    &h->s.dinv};
  for (double** p : f64) alloc((void**)p, (size_t)n * sizeof(double));
  alloc((void**)&h->s.asym, sizeof(int));
  int dev_sms = 0;
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
  h->sms = dev_sms > 0 ? dev_sms : 148;

  alloc((void**)&h->ws.part, sizeof(double) * kPartSlots * h->sms * 8);
  alloc((void**)&h->ws.counter, sizeof(unsigned long long));
  alloc((void**)&h->ws.err, sizeof(int));
  alloc((void**)&h->ws.result, sizeof(SolveResult));
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&h->res_h, sizeof(SolveResult), 0);
  for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&h->ev[i]);
  if (e != cudaSuccess) {
    set_error("eaf_cg_create", e);
    rc = (e == cudaErrorMemoryAllocation) ? EAF_ENOMEM : EAF_ECUDA;
    free_handle(h);
    delete h;
    return rc;
  }
  *out = h;
  return EAF_OK;
}

int eaf_cg_create(eaf_cg_t* out, int nr, int nth, int nz, int device) {
  return eaf_cg_create_mesh(out, nr, nth, nz, 0, device);
}

int eaf_cg_destroy(eaf_cg_t h) {
  if (!h) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->st);
  free_handle(h);
  delete h;
  return EAF_OK;
}

int eaf_cg_set_launch(eaf_cg_t h, int block_threads, int grid_blocks) {
  if (!h || block_threads < 0 || grid_blocks < 0) return EAF_EINVAL;
  if (block_threads != 0 &&
      (block_threads % 32 != 0 || block_threads > 1024 || block_threads < 64))
    return EAF_EINVAL;
  h->block = block_threads;
  h->grid = grid_blocks;
  return EAF_OK;
}

int eaf_cg_get_launch(eaf_cg_t h, int* block_threads, int* grid_blocks) {
  if (!h || !block_threads || !grid_blocks) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  pick_launch(h, true, grid_blocks, block_threads);
  return EAF_OK;
}

int eaf_cg_last_launch(eaf_cg_t h, int* block_threads, int* grid_blocks) {
  if (!h || !block_threads || !grid_blocks) return EAF_EINVAL;
  *block_threads = h->last_block;
  *grid_blocks = h->last_grid;
  return EAF_OK;
}

int eaf_cg_set_form(eaf_cg_t h, int form) {
  if (!h || (form != EAF_CG_FORM_REFERENCE && form != EAF_CG_FORM_ONE_REDUCTION))
    return EAF_EINVAL;
  h->form = form;
  return EAF_OK;
}

int eaf_cg_get_form(eaf_cg_t h, int* form) {
  if (!h || !form) return EAF_EINVAL;
  *form = h->form;
  return EAF_OK;
}

int eaf_cg_set_timeout_ms(eaf_cg_t h, double ms) {
  if (!h || !(ms > 0.0)) return EAF_EINVAL;
  h->timeout_ns = (uint64_t)(ms * 1.0e6);
  return EAF_OK;
}

int eaf_cg_last_timing(eaf_cg_t h, double* solve_ms, double* kernel_ms, int* sym,
                       int* kernels) {
  if (!h) return EAF_EINVAL;
  if (solve_ms) *solve_ms = h->last_solve_ms;
  if (kernel_ms) *kernel_ms = h->last_kernel_ms;
  if (sym) *sym = h->last_sym;
  if (kernels) *kernels = h->last_kernels;
  return EAF_OK;
}

double eaf_cg_last_e2e_ms(eaf_cg_t h) { return h ? h->last_e2e_ms : 0.0; }

void* eaf_cg_stream(eaf_cg_t h) { return h ? (void*)h->st : nullptr; }

int eaf_host_alloc(void** ptr, size_t bytes) {
  if (!ptr) return EAF_EINVAL;
  cudaError_t e = cudaHostAlloc(ptr, bytes, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    set_error("cudaHostAlloc", e);
    return EAF_ENOMEM;
  }
  return EAF_OK;
}
int eaf_host_free(void* ptr) {
  EAF_CUDA(cudaFreeHost(ptr));
  return EAF_OK;
}
int eaf_host_register(void* ptr, size_t bytes) {
  if (!ptr || !bytes) return EAF_EINVAL;
  EAF_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterPortable));
  return EAF_OK;
}
int eaf_host_unregister(void* ptr) {
  if (!ptr) return EAF_EINVAL;
  EAF_CUDA(cudaHostUnregister(ptr));
  return EAF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Solve paths
// ---------------------------------------------------------------------------
namespace {

bool any_null(const double* const* p, int n) {
  for (int i = 0; i < n; ++i)
    if (!p[i]) return true;
  return false;
}

int ensure_f32(eaf_cg* h) {
  if (h->have_f32) return EAF_OK;
  const size_t n = (size_t)h->d.n;
  float** f32[] = {&h->f.aP, &h->f.aE, &h->f.aN, &h->f.aT, &h->f.aW,
                   &h->f.aS, &h->f.aB, &h->f.r,  &h->f.z,  &h->f.q,
                   &h->f.e,  &h->f.p,  &h->f.p2};
  for (float** p : f32) {
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(float));
    if (e != cudaSuccess) {
      set_error("cudaMalloc(f32)", e);
      return EAF_ENOMEM;
    }
  }
  h->have_f32 = true;
  return EAF_OK;
}

struct SolveOpts {
  bool mixed;
  int max_iter;   // plain: max_iter; mixed: max_inner
  int max_outer;  // mixed only
  double tol, inner_tol;
};

// Device-side solve: inputs in halo layout on the device, phi written in
// place. Enqueues pack, solver, unpack on h->st; does not synchronise.
int enqueue_solve(eaf_cg* h, const HaloInputs& in, double* phi, const SolveOpts& o) {
  EAF_CUDA(cudaEventRecord(h->ev[1], h->st));
  EAF_CUDA(eaf::launch_pack_f64(h->d, in, h->s, h->st));
  int grid, block;
  if (o.mixed) {
    int rc = ensure_f32(h);
    if (rc != EAF_OK) return rc;
    pick_launch(h, false, &grid, &block);
    EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
    EAF_CUDA(eaf::launch_cg_mixed(h->d, h->s, h->f, h->ws, o.max_outer, o.max_iter,
                                  o.tol, o.inner_tol, h->timeout_ns, grid, block,
                                  h->st));
  } else {
    pick_launch(h, true, &grid, &block);
    EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
    if (h->form == EAF_CG_FORM_ONE_REDUCTION)
      EAF_CUDA(eaf::launch_cg1_f64(h->d, h->s, h->ws, o.max_iter, o.tol, h->timeout_ns,
                                   grid, block, h->st));
    else
      EAF_CUDA(eaf::launch_cg_f64(h->d, h->s, h->ws, o.max_iter, o.tol, h->timeout_ns,
                                  grid, block, h->st));
  }
  h->last_grid = grid;
  h->last_block = block;
  EAF_CUDA(cudaEventRecord(h->ev[3], h->st));
  EAF_CUDA(eaf::launch_unpack_f64(h->d, h->s.x, phi, h->st));
  EAF_CUDA(cudaEventRecord(h->ev[4], h->st));
  EAF_CUDA(cudaMemcpyAsync(h->res_h, h->ws.result, sizeof(SolveResult),
                           cudaMemcpyDeviceToHost, h->st));
  h->last_kernels = 3;
  return EAF_OK;
}

int finish_solve(eaf_cg* h, bool host_path, double* residual, int* n_iter,
                 int* n_outer) {
  EAF_CUDA(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[1], h->ev[4]) == cudaSuccess) h->last_solve_ms = ms;
  if (cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]) == cudaSuccess) h->last_kernel_ms = ms;
  if (host_path && cudaEventElapsedTime(&ms, h->ev[0], h->ev[5]) == cudaSuccess)
    h->last_e2e_ms = ms;
  const SolveResult& r = *h->res_h;
  h->last_sym = r.sym;
  if (residual) *residual = r.residual;
  if (n_iter) *n_iter = r.n_iter;
  if (n_outer) *n_outer = r.n_outer;
  return r.status;
}

int solve_device(eaf_cg* h, const double* const arr[8], double* phi,
                 const SolveOpts& o, double* residual, int* n_iter, int* n_outer) {
  if (!h || !phi || !residual || !n_iter || any_null(arr, 8)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  HaloInputs in = {arr[0], arr[1], arr[2], arr[3], arr[4], arr[5], arr[6], arr[7], phi};
  int rc = enqueue_solve(h, in, phi, o);
  if (rc != EAF_OK) return rc;
  return finish_solve(h, false, residual, n_iter, n_outer);
}

int solve_host(eaf_cg* h, const double* const arr[8], double* phi, const SolveOpts& o,
               double* residual, int* n_iter, int* n_outer) {
  if (!h || !phi || !residual || !n_iter || any_null(arr, 8)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  const size_t bytes = h->nh * sizeof(double);
  EAF_CUDA(cudaEventRecord(h->ev[0], h->st));
  for (int i = 0; i < 8; ++i)
    EAF_CUDA(cudaMemcpyAsync(h->stage[i], arr[i], bytes, cudaMemcpyHostToDevice, h->st));
  EAF_CUDA(cudaMemcpyAsync(h->stage[8], phi, bytes, cudaMemcpyHostToDevice, h->st));
  HaloInputs in = {h->stage[0], h->stage[1], h->stage[2], h->stage[3], h->stage[4],
                   h->stage[5], h->stage[6], h->stage[7], h->stage[8]};
  int rc = enqueue_solve(h, in, h->stage[8], o);
  if (rc != EAF_OK) return rc;
  EAF_CUDA(cudaMemcpyAsync(phi, h->stage[8], bytes, cudaMemcpyDeviceToHost, h->st));
  EAF_CUDA(cudaEventRecord(h->ev[5], h->st));
  return finish_solve(h, true, residual, n_iter, n_outer);
}

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

int eaf_cg_solve_f64(eaf_cg_t h, const double* aW, const double* aE, const double* aS,
                     const double* aN, const double* aB, const double* aT,
                     const double* aP, const double* Su, double* phi, int max_iter,
                     double tol, double* residual, int* n_iter) {
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  SolveOpts o = {false, max_iter, 0, tol, 0.0};
  return solve_host(h, arr, phi, o, residual, n_iter, nullptr);
}

int eaf_cg_solve_f64_device(eaf_cg_t h, const double* aW, const double* aE,
                            const double* aS, const double* aN, const double* aB,
                            const double* aT, const double* aP, const double* Su,
                            double* phi, int max_iter, double tol, double* residual,
                            int* n_iter) {
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  SolveOpts o = {false, max_iter, 0, tol, 0.0};
  return solve_device(h, arr, phi, o, residual, n_iter, nullptr);
}

int eaf_cg_solve_mixed(eaf_cg_t h, const double* aW, const double* aE, const double* aS,
                       const double* aN, const double* aB, const double* aT,
                       const double* aP, const double* Su, double* phi, int max_outer,
                       int max_inner, double tol, double inner_tol, double* residual,
                       int* n_iter, int* n_outer) {
  if (!(inner_tol > 0.0 && inner_tol < 1.0) || max_inner < 1) return EAF_EINVAL;
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  SolveOpts o = {true, max_inner, max_outer, tol, inner_tol};
  return solve_host(h, arr, phi, o, residual, n_iter, n_outer);
}

int eaf_cg_solve_mixed_device(eaf_cg_t h, const double* aW, const double* aE,
                              const double* aS, const double* aN, const double* aB,
                              const double* aT, const double* aP, const double* Su,
                              double* phi, int max_outer, int max_inner, double tol,
                              double inner_tol, double* residual, int* n_iter,
                              int* n_outer) {
  if (!(inner_tol > 0.0 && inner_tol < 1.0) || max_inner < 1) return EAF_EINVAL;
  const double* arr[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  SolveOpts o = {true, max_inner, max_outer, tol, inner_tol};
  return solve_device(h, arr, phi, o, residual, n_iter, n_outer);
}

// ---------------------------------------------------------------------------
// Barrier self-test: two blocks wait on a counter that only reaches half of
// its target, so every wait runs into its bound and the kernel reports
// EAF_ETIMEOUT through the error word; the context stays usable.
// ---------------------------------------------------------------------------
int eaf_selftest_barrier_timeout(int device, double timeout_ms) {
  if (!(timeout_ms > 0.0) || timeout_ms > 10000.0) return EAF_EINVAL;
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) return EAF_ECUDA;
  GroupWs ws = {};
  cudaStream_t st = nullptr;
  int err_h = 0;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.part, sizeof(double) * 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.counter, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.err, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.result, sizeof(SolveResult));
  if (e == cudaSuccess)
    e = eaf::launch_barrier_selftest(ws, (uint64_t)(timeout_ms * 1.0e6), st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&err_h, ws.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(ws.part);
  cudaFree(ws.counter);
  cudaFree(ws.err);
  cudaFree(ws.result);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    set_error("selftest", e);
    return EAF_ECUDA;
  }
  return err_h;
}

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

namespace eaf {
namespace {
// Two blocks; the group is declared with three members, so the arrival
// target of the first barrier is never reached and both waits expire.
__global__ void barrier_selftest_kernel(GroupWs ws, uint64_t timeout_ns) {
  Group g;
  g.counter = ws.counter;
  g.err = ws.err;
  g.part = ws.part;
  g.stage = group_stage_smem();
  g.nb = 3;
  g.bid = blockIdx.x;
  g.timeout_ns = timeout_ns;
  g.epoch = 0;
  group_barrier(g);
}
}  // namespace

cudaError_t launch_barrier_selftest(const GroupWs& ws, uint64_t timeout_ns,
                                    cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  void* args[] = {(void*)&ws, (void*)&timeout_ns};
  return cudaLaunchCooperativeKernel((const void*)barrier_selftest_kernel, dim3(2),
                                     dim3(64), args, 0, st);
}
}  // namespace eaf
