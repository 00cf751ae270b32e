// Diagnostics: the cost of one group all-reduce (block reduction, group
// barrier, staging and fold of the block partials) on its own, for the
// launch shapes the solvers use. Feeds the launch-shape choice and the
// latency accounting of the solver iteration.
#include <cuda_runtime.h>

#include "cg_kernels.h"
#include "eafcg.h"
#include "eafcg_internal.h"

namespace eaf {
namespace {

template <int FORM>
__global__ void allreduce_bench_kernel(GroupWs ws, int iters, uint64_t timeout_ns,
                                       double* out) {
  Group g;
  g.counter = ws.counter;
  g.err = ws.err;
  g.part = ws.part;
  g.stage = group_stage_smem();
  g.nb = gridDim.x;
  g.bid = blockIdx.x;
  g.timeout_ns = timeout_ns;
  g.epoch = 0;
  double acc = 0.0;
  for (int it = 0; it < iters; ++it) {
    double v[2] = {(double)(threadIdx.x + it), 1.0};
    if (!group_allsum<2, double, FORM>(v, g, (it & 1) ? 2 : 0)) break;
    acc = acc + v[0] * v[1];
  }
  if (g.bid == 0 && threadIdx.x == 0) *out = acc;
}

}  // namespace
}  // namespace eaf

extern "C" int eaf_diag_allreduce_us(int device, int blocks, int threads, int iters,
                                     int form, double* us_per_allreduce) {
  if (!us_per_allreduce || blocks < 1 || blocks > eaf::kMaxGroupBlocks ||
      threads < 64 || threads > 1024 || threads % 32 || iters < 1 || form < 0 ||
      form > 3)
    return EAF_EINVAL;
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) return EAF_ECUDA;
  eaf::GroupWs ws = {};
  double* out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.part, sizeof(double) * 4 * blocks);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.counter, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ws.err, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&out, sizeof(double));
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const void* kern = form == 0   ? (const void*)eaf::allreduce_bench_kernel<0>
                     : form == 1 ? (const void*)eaf::allreduce_bench_kernel<1>
                     : form == 2 ? (const void*)eaf::allreduce_bench_kernel<2>
                                 : (const void*)eaf::allreduce_bench_kernel<3>;
  uint64_t timeout = 2000ull * 1000ull * 1000ull;
  float ms = 0.f;
  for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // rep 0 warms up
    e = cudaMemsetAsync(ws.counter, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws.err, 0, sizeof(int), st);
    void* args[] = {(void*)&ws, (void*)&iters, (void*)&timeout, (void*)&out};
    if (e == cudaSuccess) e = cudaEventRecord(e0, st);
    if (e == cudaSuccess)
      e = cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(threads), args, 0, st);
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  }
  int err_h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&err_h, ws.err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(ws.part);
  cudaFree(ws.counter);
  cudaFree(ws.err);
  cudaFree(out);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_diag_allreduce_us", e);
    return EAF_ECUDA;
  }
  *us_per_allreduce = 1.0e3 * ms / iters;
  return err_h;
}

extern "C" int eaf_diag_div_check(int device, long long n, unsigned long long seed,
                                  long long* mismatches, long long* fast_path) {
  if (n < 1 || !mismatches || !fast_path) return EAF_EINVAL;
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) return EAF_ECUDA;
  unsigned long long* d = nullptr;
  unsigned long long h[2] = {0, 0};
  cudaError_t e = cudaMalloc((void**)&d, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = eaf::run_div_check(n, seed, d, 0);
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_diag_div_check", e);
    return EAF_ECUDA;
  }
  *mismatches = (long long)h[0];
  *fast_path = (long long)h[1];
  return EAF_OK;
}
