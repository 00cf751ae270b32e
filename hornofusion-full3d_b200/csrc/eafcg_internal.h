// Host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "cg_kernels.h"


namespace eaf {

// Records the last CUDA failure of this thread for eaf_last_error().
void set_error(const char* what, cudaError_t e);
// Records a plain message (no CUDA error) for eaf_last_error().
void set_error_text(const char* msg);

// Makes `dev` current for the lifetime of the guard and restores the
// caller's device afterwards.
class DeviceGuard {
 public:
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
  bool ok() const { return ok_; }

 private:
  int prev_;
  bool ok_;
};


// ---- batched-launch planning (batch.cu), shared with the server ----------
// Lane tables of one batched launch over `grid` blocks.
struct LanePlan {
  std::vector<int> lane_of_block, lane_first, lane_width, q_begin, queue;
  std::vector<int> packed() const;  // device table order (BatchTables)
};
// Co-resident blocks of 512 threads for the batch kernels on `device`.
int batch_capacity(int device, int* blocks);
// Lanes for systems of the given lane widths and cell counts on G blocks.
int plan_lanes(const std::vector<int>& widths, const std::vector<long long>& cells,
               int G, LanePlan* out);
// Modelled solve time (us) of one system of `cells` cells on w blocks.
double model_solve_us(long long cells, int w);
BatchTables tables_from(const int* d_tab, int grid, int nlanes, const BatchSys* d_sys,
                        unsigned long long* counters, double* parts, int* err);

}  // namespace eaf
