// C-ABI shim of libeafcg.so: handle lifetime, device buffers, uploads,
// launches, result readback and timing for the single-system CG solvers
// (the other solvers on the same handle are in api_pressure.cu). The public
// contract is documented in include/eafcg.h.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <new>

#include "cg_kernels.h"
#include "cluster_red.cuh"
#include "eafcg.h"
#include "eafcg_internal.h"
#include "handle.h"
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
// Doubles of a handle's partial table (also the slot table of the cluster
// all-reduce).
inline size_t kPartTableDoubles(const eaf_cg* h) { return (size_t)kPartSlots * h->sms * 8; }
constexpr uint64_t kDefaultTimeoutNs = 2000ull * 1000ull * 1000ull;

}  // namespace

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
  cudaFree(h->trace_d);
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

namespace eaf {

std::mutex& launch_attr_mutex() {
  static std::mutex m;
  return m;
}

// Launch shape for a persistent kernel over n cells: an explicit
// eaf_cg_set_launch shape, else the tuned shape of this mesh (FP64 solver),
// else, for the reference-form FP64 solver on a mesh that fits, one
// cluster-resident launch (below), else one 1024-thread block up to 8192
// cells or one 512-thread block per 2048 cells; capped by co-residency of
// the kernel (variant) that runs blocks of that size. The reference-form FP64 solver may run on a grid of
// thread-block clusters (eaf_cg_set_cluster, else the tuned cluster size):
// the grid is then a whole number of clusters, at most as many as can be
// resident; a cluster size the device cannot launch falls back to none.
SolverLaunch choose_launch(int nr, int nth, int nz, int sms, int req_block, int req_grid,
                           int req_cluster, int form, bool f64, int req_kernel) {
  const long long n = (long long)nr * nth * nz;
  auto kernel_for = [f64, form, n](int b) {
    if (!f64) return cg_mixed_kernel_ptr();
    return form == EAF_CG_FORM_ONE_REDUCTION ? cg1_f64_kernel_ptr(b) : cg_f64_kernel_ptr(b, n);
  };
  int b = req_block > 0 ? req_block : kDefaultBlock;
  int g;
  int tb = 0, tg = 0, tc = 1, ts = 0;
  const bool automatic = req_block == 0 && req_grid == 0;
  const bool tuned = automatic && f64 && tuned_single_launch(nr, nth, nz, &tb, &tg, &tc, &ts);
  if (tuned) {
    b = tb;
    g = tg;
  } else if (req_grid > 0) {
    g = req_grid;
  } else if (n <= 8192) {
    b = req_block > 0 ? req_block : 1024;
    g = 1;
  } else {
    long long want = (n + (long long)b * 4 - 1) / ((long long)b * 4);
    g = (int)(want < 1 ? 1 : want);
  }
  int c = 1;
  if (automatic && f64 && form == EAF_CG_FORM_REFERENCE && !tuned && req_cluster == 0) {
    // A small mesh outside the table: one cluster that keeps the system in
    // its shared memory (8 blocks up to 8192 cells, else 16), one cell per
    // thread up to 640 cells a block, else two.
    const int cs = n <= 8192 ? 8 : 16;
    const long long per = (n + cs - 1) / cs;
    long long t = per <= 640 ? per : (per + 1) / 2;
    t = ((t + 31) / 32) * 32;
    const int bs = (int)(t < 64 ? 64 : (t > 1024 ? 1024 : t));
    if (dsm_can_launch(n, bs, cs) && max_active_clusters(bs, n, cs) >= 1) {
      b = bs;
      g = cs;
      tc = cs;
    }
  }
  if (f64 && form == EAF_CG_FORM_REFERENCE) {
    c = req_cluster > 0 ? req_cluster : (automatic ? tc : 1);
    if (c > 1) {
      const int active = max_active_clusters(b, n, c);
      if (active < 1) {
        c = 1;
      } else {
        if (g < c) g = c;
        g -= g % c;
        int ncl = g / c;
        if (ncl > active) ncl = active;
        if (ncl > kMaxClusters) ncl = kMaxClusters;
        g = ncl * c;
      }
    }
  }
  int stream = 0, slots = 0, keep = 0;
  if (f64 && form == EAF_CG_FORM_REFERENCE && c == 1) {
    int k = req_kernel;
    if (k == EAF_CG_KERNEL_AUTO)
      k = !automatic ? EAF_CG_KERNEL_LOADS
          : ts == 2  ? EAF_CG_KERNEL_KEEP
          : ts == 1  ? EAF_CG_KERNEL_STREAM
                     : EAF_CG_KERNEL_LOADS;
    slots = k == EAF_CG_KERNEL_SLOTS;
    stream = k == EAF_CG_KERNEL_STREAM;
    keep = k == EAF_CG_KERNEL_KEEP;
    if (stream && (b % 32 != 0 || stream_max_coresident(b, nr, sms) < 1)) stream = 0;
  }
  if (c == 1) {
    const int cap = stream ? stream_max_coresident(b, nr, sms)
                           : max_coresident(kernel_for(b), b, sms);
    if (cap > 0 && g > cap) g = cap;
    if (g > sms * 8) g = sms * 8;
  }
  // The kept slices must fit the shared memory of blocks that are all
  // resident at once; otherwise the per-thread-load kernel runs.
  if (keep && keep_max_coresident(b, n, g, sms) < g) keep = 0;
  SolverLaunch L;
  L.grid = g;
  L.block = b;
  L.cluster = c;
  L.stream = stream;
  L.slots = slots;
  L.keep = keep;
  if (slots && g > kMaxClusters) L.grid = kMaxClusters;
  return L;
}

bool runs_resident(const SolverLaunch& L, long long n, bool allowed) {
  return allowed && L.cluster > 1 && L.grid == L.cluster &&
         dsm_can_launch(n, L.block, L.cluster);
}

cudaError_t launch_f64_solver(const SolverLaunch& L, int resident, const MeshDims& d,
                              const SysF64& s, const GroupWs& ws, size_t slot_doubles,
                              int max_iter, double tol, uint64_t timeout_ns, cudaStream_t st) {
  if (runs_resident(L, d.n, resident != 0))
    return launch_cg_f64_dsm(d, s, ws, max_iter, tol, L.block, L.cluster, st,
                             resident == 2 ? kDsmSignalMbarrier : kDsmSignalClusterBarrier,
                             timeout_ns);
  if (L.cluster > 1 || L.slots)
    return launch_cg_f64_cluster(d, s, ws, ws.part, slot_doubles, max_iter, tol, timeout_ns,
                                 L.grid, L.block, L.cluster, st);
  if (L.stream)
    return launch_cg_f64_stream(d, s, ws, max_iter, tol, timeout_ns, L.grid, L.block, st);
  if (L.keep)
    return launch_cg_f64_keep(d, s, ws, max_iter, tol, timeout_ns, L.grid, L.block, st);
  return launch_cg_f64(d, s, ws, max_iter, tol, timeout_ns, L.grid, L.block, st);
}

}  // namespace eaf

static eaf::SolverLaunch pick_launch(const eaf_cg* h, bool f64, int* grid, int* block,
                                     int* cluster) {
  const eaf::SolverLaunch L = eaf::choose_launch(h->nr, h->nth, h->nz, h->sms, h->block,
                                                 h->grid, h->cluster, h->form, f64,
                                                 h->kernel);
  *grid = L.grid;
  *block = L.block;
  *cluster = L.cluster;
  return L;
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
  h->resident = 1;
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
  // One padding cell (two, rounded) past each compact array: the streaming
  // kernel's bulk copies move whole 16-byte pairs of cells.
  for (double** p : f64) alloc((void**)p, (size_t)(n + 2) * sizeof(double));
  alloc((void**)&h->s.asym, sizeof(int));
  int dev_sms = 0;
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
  h->sms = dev_sms > 0 ? dev_sms : 148;

  alloc((void**)&h->ws.part, sizeof(double) * kPartTableDoubles(h));
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
  int cluster = 1;
  pick_launch(h, true, grid_blocks, block_threads, &cluster);
  return EAF_OK;
}

int eaf_cg_last_launch(eaf_cg_t h, int* block_threads, int* grid_blocks) {
  if (!h || !block_threads || !grid_blocks) return EAF_EINVAL;
  *block_threads = h->last_block;
  *grid_blocks = h->last_grid;
  return EAF_OK;
}

int eaf_cg_set_cluster(eaf_cg_t h, int cluster_blocks) {
  if (!h || cluster_blocks < 0 || cluster_blocks > eaf::kMaxClusterSize) return EAF_EINVAL;
  h->cluster = cluster_blocks;
  return EAF_OK;
}

int eaf_cg_get_cluster(eaf_cg_t h, int* cluster_blocks) {
  if (!h || !cluster_blocks) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  int grid = 0, block = 0;
  pick_launch(h, true, &grid, &block, cluster_blocks);
  return EAF_OK;
}

int eaf_cg_mixed_trace(eaf_cg_t h, double* steps, int max_steps, int* n_steps) {
  if (!h || !n_steps || max_steps < 0 || (max_steps > 0 && !steps)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  int n = h->res_h ? h->res_h->n_outer : 0;
  if (n > h->trace_cap) n = h->trace_cap;
  if (n > max_steps) n = max_steps;
  *n_steps = n;
  if (n > 0)
    EAF_CUDA(cudaMemcpy(steps, h->trace_d, sizeof(double) * 3 * (size_t)n,
                        cudaMemcpyDeviceToHost));
  return EAF_OK;
}

int eaf_cg_set_kernel(eaf_cg_t h, int kernel) {
  if (!h || kernel < EAF_CG_KERNEL_AUTO || kernel > EAF_CG_KERNEL_KEEP) return EAF_EINVAL;
  h->kernel = kernel;
  return EAF_OK;
}

int eaf_cg_last_kernel(eaf_cg_t h, int* kernel) {
  if (!h || !kernel) return EAF_EINVAL;
  *kernel = h->last_stream == 3   ? EAF_CG_KERNEL_KEEP
            : h->last_stream == 2 ? EAF_CG_KERNEL_SLOTS
            : h->last_stream      ? EAF_CG_KERNEL_STREAM
                                  : EAF_CG_KERNEL_LOADS;
  return EAF_OK;
}

int eaf_cg_set_resident(eaf_cg_t h, int resident) {
  if (!h || resident < 0 || resident > 2) return EAF_EINVAL;
  h->resident = resident;
  return EAF_OK;
}

int eaf_cg_last_cluster(eaf_cg_t h, int* cluster_blocks) {
  if (!h || !cluster_blocks) return EAF_EINVAL;
  *cluster_blocks = h->last_cluster > 0 ? h->last_cluster : 1;
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
// Solve paths (shared with api_pressure.cu through handle.h)
// ---------------------------------------------------------------------------
bool any_null(const double* const* p, int n) {
  for (int i = 0; i < n; ++i)
    if (!p[i]) return true;
  return false;
}

static int ensure_f32(eaf_cg* h) {
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


// Device-side solve: inputs in halo layout on the device, phi written in
// place. Enqueues pack, solver, unpack on h->st; does not synchronise.
int enqueue_solve(eaf_cg* h, const HaloInputs& in, double* phi, const SolveOpts& o) {
  EAF_CUDA(cudaEventRecord(h->ev[1], h->st));
  EAF_CUDA(eaf::launch_pack_f64(h->d, in, h->s, h->st));
  int grid, block, cluster = 1;
  if (o.mixed) {
    int rc = ensure_f32(h);
    if (rc != EAF_OK) return rc;
    pick_launch(h, false, &grid, &block, &cluster);
    if (o.max_outer > h->trace_cap) {
      cudaFree(h->trace_d);
      h->trace_d = nullptr;
      h->trace_cap = 0;
      EAF_CUDA(cudaMalloc((void**)&h->trace_d, sizeof(double) * 3 * (size_t)o.max_outer));
      h->trace_cap = o.max_outer;
    }
    EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
    EAF_CUDA(eaf::launch_cg_mixed(h->d, h->s, h->f, h->ws, o.max_outer, o.max_iter,
                                  o.tol, o.inner_tol, h->timeout_ns, grid, block,
                                  h->st, h->trace_d));
  } else {
    const eaf::SolverLaunch L = pick_launch(h, true, &grid, &block, &cluster);
    h->last_stream = L.keep ? 3 : L.slots ? 2 : L.stream;
    EAF_CUDA(cudaEventRecord(h->ev[2], h->st));
    if (h->form == EAF_CG_FORM_ONE_REDUCTION)
      EAF_CUDA(eaf::launch_cg1_f64(h->d, h->s, h->ws, o.max_iter, o.tol, h->timeout_ns,
                                   grid, block, h->st));
    else
      EAF_CUDA(eaf::launch_f64_solver(L, h->resident, h->d, h->s, h->ws,
                                      kPartTableDoubles(h), o.max_iter, o.tol,
                                      h->timeout_ns, h->st));
  }
  h->last_grid = grid;
  h->last_block = block;
  h->last_cluster = cluster;
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

static int solve_device(eaf_cg* h, const double* const arr[8], double* phi,
                 const SolveOpts& o, double* residual, int* n_iter, int* n_outer) {
  if (!h || !phi || !residual || !n_iter || any_null(arr, 8)) return EAF_EINVAL;
  eaf::DeviceGuard guard(h->device);
  HaloInputs in = {arr[0], arr[1], arr[2], arr[3], arr[4], arr[5], arr[6], arr[7], phi};
  int rc = enqueue_solve(h, in, phi, o);
  if (rc != EAF_OK) return rc;
  return finish_solve(h, false, residual, n_iter, n_outer);
}

static int solve_host(eaf_cg* h, const double* const arr[8], double* phi, const SolveOpts& o,
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

int eaf_selftest_allreduce_timeout(int device, double timeout_ms, int mode) {
  if (!(timeout_ms > 0.0) || timeout_ms > 10000.0 || (mode != 0 && mode != 1))
    return EAF_EINVAL;
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) return EAF_ECUDA;
  GroupWs ws = {};
  cudaStream_t st = nullptr;
  int err_h = 0;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.part, sizeof(double) * 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.counter, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.err, sizeof(int));
  if (e == cudaSuccess)
    e = eaf::launch_allreduce_selftest(ws, (uint64_t)(timeout_ms * 1.0e6), mode, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&err_h, ws.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(ws.part);
  cudaFree(ws.counter);
  cudaFree(ws.err);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    set_error("selftest", e);
    return EAF_ECUDA;
  }
  return err_h;
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
