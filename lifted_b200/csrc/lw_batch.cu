// Instantiations and launch wrappers of the persistent batch kernel.
#include <cuda_runtime.h>

#include "lw_batch.hpp"
#include "lw_batch_kernel.cuh"
#include "lw_launch.hpp"

namespace lw {

namespace {

template <typename T>
cudaError_t configure(int dev) {
  static bool done[kMaxDevices] = {};
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (done[dev]) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(
      batch_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxDynSmem);
  if (e != cudaSuccess) return e;
  done[dev] = true;
  return cudaSuccess;
}

template <typename T>
cudaError_t launch_impl(const BatchParams<T>& p, int grid, int block,
                        size_t smem, cudaStream_t stream) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = configure<T>(dev);
  if (e != cudaSuccess) return e;
  batch_kernel<T><<<grid, block, smem, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_batch(const BatchParams<float>& p, int grid, int block,
                         size_t smem, cudaStream_t stream) {
  return launch_impl(p, grid, block, smem, stream);
}
cudaError_t launch_batch(const BatchParams<double>& p, int grid, int block,
                         size_t smem, cudaStream_t stream) {
  return launch_impl(p, grid, block, smem, stream);
}

int batch_occupancy(int dtype_bytes, int block, size_t smem) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  int n = 0;
  cudaError_t e;
  if (dtype_bytes == 4) {
    if (configure<float>(dev) != cudaSuccess) return 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<float>, block, smem);
  } else {
    if (configure<double>(dev) != cudaSuccess) return 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<double>, block, smem);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace lw
