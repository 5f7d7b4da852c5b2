// Host-visible launch interface of the CUDA kernels (implemented in
// lw_kernels.cu and friends).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "lw_types.hpp"

namespace lw {

// Dynamic shared memory the line kernel may request (B200: 227 KB opt-in per
// block, less the kernel's static arrays).
constexpr int kMaxDevices = 64;
constexpr size_t kMaxDynSmem = 227 * 1024 - 2 * 64 * 8 - 256;

template <typename T>
struct CopyParams {
  const T* in;
  T* out;
  int64_t total;
  int32_t ndim;
  int32_t pad_;
  int64_t shape[MAX_NDIM];  // fastest-varying first
  int64_t sin[MAX_NDIM];
  int64_t sout[MAX_NDIM];
};

cudaError_t launch_line(const LineParams<float>& p, int grid, int block,
                        size_t smem, cudaStream_t stream);
cudaError_t launch_line(const LineParams<double>& p, int grid, int block,
                        size_t smem, cudaStream_t stream);
cudaError_t launch_copy(const CopyParams<float>& p, cudaStream_t stream);

// Stream-ordered scratch allocation from the current device's default memory
// pool.  The first call on a device raises the pool's release threshold so
// freed scratch stays cached in the pool across synchronisations instead of
// going back to the driver (a process-local pool attribute).
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream);
cudaError_t scratch_free(void* p, cudaStream_t stream);
cudaError_t launch_copy(const CopyParams<double>& p, cudaStream_t stream);

}  // namespace lw
