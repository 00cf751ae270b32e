// The solver handle and the host helpers shared by the C-ABI translation
// units (api.cu: handles and the CG; api_pressure.cu: the other solvers and
// the pressure step on the same handle).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cg_kernels.h"
#include "eafcg.h"
#include "eafcg_internal.h"

struct eaf_cg {
  int nr, nth, nz, device;
  eaf::MeshDims d;
  size_t nh;  // halo-layout elements per array
  cudaStream_t st;
  double* stage[9];  // aW aE aS aN aB aT aP Su phi, halo layout (host path)
  eaf::SysF64 s;
  eaf::SysF32 f;
  bool have_f32;
  eaf::GroupWs ws;
  eaf::SolveResult* res_h;  // pinned
  int block, grid;     // 0 = automatic
  int cluster;         // blocks per thread-block cluster; 0 = automatic, 1 = none
  int resident;        // one-cluster launches keep the system in shared memory
  int kernel;          // EAF_CG_KERNEL_*: per-thread loads or bulk-copy streaming
  int last_stream;     // the last FP64 solve's flat kernel: 0 loads, 1 stream, 2 slots, 3 keep
  double* trace_d;     // mixed form: per refinement step trace (lazy)
  int trace_cap;       // refinement steps trace_d holds
  int sms;
  uint64_t timeout_ns;
  cudaEvent_t ev[6];   // e2e0, solve0, kern0, kern1, solve1, e2e1
  double last_solve_ms, last_kernel_ms, last_e2e_ms;
  int last_sym, last_kernels;
  int last_grid, last_block, last_cluster;
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

// Returns EAF_ECUDA from the enclosing function, recording the failure for
// eaf_last_error(), when `call` does not return cudaSuccess.
#define EAF_CUDA(call)                     \
  do {                                     \
    cudaError_t e_ = (call);               \
    if (e_ != cudaSuccess) {               \
      eaf::set_error(#call, e_);           \
      return EAF_ECUDA;                    \
    }                                      \
  } while (0)

struct SolveOpts {
  bool mixed;
  int max_iter;   // plain: max_iter; mixed: max_inner
  int max_outer;  // mixed only
  double tol, inner_tol;
};

// True if any of the n pointers is null.
bool any_null(const double* const* p, int n);
// Enqueues pack, the FP64 or mixed solver and unpack on h->st (no sync).
int enqueue_solve(eaf_cg* h, const eaf::HaloInputs& in, double* phi, const SolveOpts& o);
// Synchronises h->st, records the timings and returns the solve's status.
int finish_solve(eaf_cg* h, bool host_path, double* residual, int* n_iter, int* n_outer);
