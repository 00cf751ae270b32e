// Host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>


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


}  // namespace eaf
