// eaf_cg_solve_f64_noalloc: the plain FP64 solve for callers that must not
// allocate device memory.
//
// Who cannot allocate, and why: a simulator whose device memory is owned end
// to end by its own pool allocator or fixed budget (a cudaMalloc behind its
// back either fails or fragments that pool), and code on a latency-critical
// path, where cudaMalloc/cudaFree would synchronise the device and stall
// every other stream. Such a caller owns its inputs and phi and hands them
// over; everything else this solve needs lives in one file-scope device
// array that each GPU holds from library load until process exit.
//
// Limits and sharing rules:
//   * at most kNoallocMaxCells = EAF_NOALLOC_MAX_CELLS interior cells
//     (32768; 18x36x24 fits, 35x70x50 does not); larger meshes are refused
//     with EAF_EINVAL and an explanatory eaf_last_error() text;
//   * the array is shared by every call on a device and keeps the previous
//     call's contents; each call re-packs the inputs and zeroes the barrier
//     counter, the error word and the symmetry flag before its solver runs;
//   * two calls whose work overlaps on the same GPU (different host threads,
//     or different streams not ordered by the caller) race on the array.
//     Callers serialise their calls per device;
//   * the first call on a device looks the array's device address up with
//     cudaGetSymbolAddress (with that device current) and keeps it for the
//     later calls; a lookup that fails is not kept, so the next call tries
//     again. That first call should come before any stream capture begins
//     on the device.
// The kernels are the ones eaf_cg_solve_f64_device runs (pack, the
// persistent CG, unpack), launched with the same default shape, so results
// are bit-identical to that entry point on the same inputs.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <mutex>

#include "cg_kernels.h"
#include "cluster_red.cuh"
#include "eafcg.h"
#include "eafcg_internal.h"
#include "tune_table.h"

namespace {

constexpr int kNoallocMaxCells = EAF_NOALLOC_MAX_CELLS;
// Blocks of the largest launch this entry makes; the partial table is sized
// for it. Every launch shape the handle entries pick for a mesh of at most
// kNoallocMaxCells cells must fit, or the two would not give the same bits:
// the tuned shapes (checked here), the small-mesh fallback of one cluster
// of at most 16 blocks, and the fallback without clusters of one 512-thread
// block per 2048 cells (checked here).
constexpr int kNoallocMaxBlocks = 64;
static_assert(eaf::max_tuned_grid_up_to(kNoallocMaxCells) <= kNoallocMaxBlocks,
              "a tuned launch for a mesh within the no-allocation limit has more "
              "blocks than the static scratch holds partials for");
static_assert((kNoallocMaxCells + 2047) / 2048 <= kNoallocMaxBlocks,
              "the fallback launch shape exceeds the static scratch's block limit");
constexpr int kPartSlots = 8;
// A cluster launch uses the partial table as its slot table: at most
// kNoallocMaxBlocks / 2 clusters of two or more blocks.
static_assert(eaf::cluster_slot_doubles(kNoallocMaxBlocks / 2) <=
                  (size_t)kPartSlots * kNoallocMaxBlocks,
              "the partial table cannot hold the cluster all-reduce's slots");
constexpr int kMaxDevices = 64;
constexpr uint64_t kNoallocTimeoutNs = 2000ull * 1000ull * 1000ull;

// Scratch layout (doubles unless stated):
//   14 compact arrays of kNoallocMaxCells: aP aE aN aT aW aS aB b x r p q p2 z
//   partial table: kPartSlots * kNoallocMaxBlocks
//   barrier counter (u64), error word (int), symmetry flag (int), result
constexpr size_t kArrays = 14;
constexpr size_t kPartOff = kArrays * kNoallocMaxCells;
constexpr size_t kCounterOff = kPartOff + (size_t)kPartSlots * kNoallocMaxBlocks;
constexpr size_t kErrOff = kCounterOff + 1;    // one double slot each
constexpr size_t kAsymOff = kErrOff + 1;
constexpr size_t kResultOff = kAsymOff + 1;
constexpr size_t kScratchDoubles =
    kResultOff + (sizeof(eaf::SolveResult) + sizeof(double) - 1) / sizeof(double);

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct DeviceSlot {
  std::mutex mu;
  double* base = nullptr;  // set once a lookup has succeeded
};
DeviceSlot g_slots[kMaxDevices];

// Device address of the scratch array on the current device `dev`. Only a
// successful lookup is kept; after a failure the next call looks again.
cudaError_t scratch_on(int dev, double** out) {
  DeviceSlot& s = g_slots[dev];
  std::lock_guard<std::mutex> lock(s.mu);
  if (!s.base) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      *out = nullptr;
      return e != cudaSuccess ? e : cudaErrorInvalidSymbol;
    }
    s.base = static_cast<double*>(p);
  }
  *out = s.base;
  return cudaSuccess;
}

}  // namespace

extern "C" int eaf_cg_solve_f64_noalloc(int nr, int nth, int nz, int device,
                                        void* stream, const double* aW,
                                        const double* aE, const double* aS,
                                        const double* aN, const double* aB,
                                        const double* aT, const double* aP,
                                        const double* Su, double* phi, int max_iter,
                                        double tol, double* residual, int* n_iter) {
  if (!aW || !aE || !aS || !aN || !aB || !aT || !aP || !Su || !phi || !residual ||
      !n_iter || nr < 1 || nth < 1 || nz < 1 || device < 0 || device >= kMaxDevices)
    return EAF_EINVAL;
  const long long n = (long long)nr * nth * nz;
  if (n > kNoallocMaxCells) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "eaf_cg_solve_f64_noalloc: %lld cells exceed the %d-cell static "
             "scratch; use eaf_cg_create/eaf_cg_solve_f64_device",
             n, kNoallocMaxCells);
    eaf::set_error_text(msg);
    return EAF_EINVAL;
  }
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) {
    eaf::set_error("eaf_cg_solve_f64_noalloc: cudaSetDevice", cudaErrorInvalidDevice);
    return EAF_ECUDA;
  }
  double* base = nullptr;
  cudaError_t e = scratch_on(device, &base);
  if (e != cudaSuccess || !base) {
    eaf::set_error("eaf_cg_solve_f64_noalloc: cudaGetSymbolAddress", e);
    return EAF_ECUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const eaf::MeshDims d = eaf::make_dims(nr, nth, nz);
  const size_t M = kNoallocMaxCells;
  eaf::SysF64 s;
  s.aP = base + 0 * M;
  s.aE = base + 1 * M;
  s.aN = base + 2 * M;
  s.aT = base + 3 * M;
  s.aW = base + 4 * M;
  s.aS = base + 5 * M;
  s.aB = base + 6 * M;
  s.b = base + 7 * M;
  s.x = base + 8 * M;
  s.r = base + 9 * M;
  s.p = base + 10 * M;
  s.q = base + 11 * M;
  s.p2 = base + 12 * M;
  s.z = base + 13 * M;
  s.s0 = s.s1 = s.dinv = nullptr;  // the single-reduction form is not launched here
  s.asym = reinterpret_cast<int*>(base + kAsymOff);
  eaf::GroupWs ws;
  ws.part = base + kPartOff;
  ws.counter = reinterpret_cast<unsigned long long*>(base + kCounterOff);
  ws.err = reinterpret_cast<int*>(base + kErrOff);
  ws.result = reinterpret_cast<eaf::SolveResult*>(base + kResultOff);

  // Launch: the default of eaf_cg_create handles on this mesh (tuned shape,
  // cluster size and resident kernel included), so that results match the
  // handle entry points bit for bit.
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_cg_solve_f64_noalloc: cudaDeviceGetAttribute", e);
    return EAF_ECUDA;
  }
  const eaf::SolverLaunch L =
      eaf::choose_launch(nr, nth, nz, sms, 0, 0, 0, EAF_CG_FORM_REFERENCE, true);
  if (L.grid > kNoallocMaxBlocks) {  // excluded by the static_asserts above
    eaf::set_error_text("eaf_cg_solve_f64_noalloc: launch shape exceeds the static scratch");
    return EAF_EINVAL;
  }

  eaf::HaloInputs in = {aW, aE, aS, aN, aB, aT, aP, Su, phi};
  e = eaf::launch_pack_f64(d, in, s, st);
  if (e == cudaSuccess)
    e = eaf::launch_f64_solver(L, 1, d, s, ws, (size_t)kPartSlots * kNoallocMaxBlocks,
                               max_iter, tol, kNoallocTimeoutNs, st);
  if (e == cudaSuccess) e = eaf::launch_unpack_f64(d, s.x, phi, st);
  eaf::SolveResult r;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&r, ws.result, sizeof(r), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_cg_solve_f64_noalloc", e);
    return EAF_ECUDA;
  }
  *residual = r.residual;
  *n_iter = r.n_iter;
  return r.status;
}
