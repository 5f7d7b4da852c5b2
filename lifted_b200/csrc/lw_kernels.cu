// Kernel instantiations and launch wrappers of the B200 lifting DWT.
#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_line_kernel.cuh"

namespace lw {

namespace {

// Generic strided nD copy (the reverse-stepping non-separable driver copies
// in -> out before working in place, src/lifted-drivers-inl.hpp:542-567).
template <typename T>
__global__ void copy_kernel(const __grid_constant__ CopyParams<T> p) {
  pdl_wait();  // the previous kernel's results (no global access before)
  pdl_trigger();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
       li < p.total; li += stride) {
    int64_t r = li, oi = 0, oo = 0;
    for (int d = 0; d < p.ndim; ++d) {
      int64_t q = r / p.shape[d];
      int64_t idx = r - q * p.shape[d];
      r = q;
      oi += idx * p.sin[d];
      oo += idx * p.sout[d];
    }
    p.out[oo] = p.in[oi];
  }
}

template <typename T>
cudaError_t launch_line_impl(const LineParams<T>& p, int grid, int block,
                             size_t smem, cudaStream_t stream) {
  static bool configured[kMaxDevices] = {};  // per instantiation, device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!configured[dev]) {
    e = cudaFuncSetAttribute(line_kernel<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kMaxDynSmem);
    if (e != cudaSuccess) return e;
    configured[dev] = true;
  }
  return launch_overlapped(line_kernel<T>, grid, block, smem, stream, p);
}

}  // namespace

cudaError_t launch_line(const LineParams<float>& p, int grid, int block,
                        size_t smem, cudaStream_t stream) {
  return launch_line_impl(p, grid, block, smem, stream);
}
cudaError_t launch_line(const LineParams<double>& p, int grid, int block,
                        size_t smem, cudaStream_t stream) {
  return launch_line_impl(p, grid, block, smem, stream);
}

cudaError_t launch_copy(const CopyParams<float>& p, cudaStream_t stream) {
  int grid = (int)((p.total + 255) / 256);
  if (grid > 148 * 16) grid = 148 * 16;
  if (grid < 1) grid = 1;
  return launch_overlapped(copy_kernel<float>, grid, 256, 0, stream, p);
}
cudaError_t launch_copy(const CopyParams<double>& p, cudaStream_t stream) {
  int grid = (int)((p.total + 255) / 256);
  if (grid > 148 * 16) grid = 148 * 16;
  if (grid < 1) grid = 1;
  return launch_overlapped(copy_kernel<double>, grid, 256, 0, stream, p);
}

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream) {
  static bool pool_ready[kMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kMaxDevices && !pool_ready[dev]) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    pool_ready[dev] = true;
  }
  return cudaMallocAsync(p, bytes, stream);
}

cudaError_t scratch_free(void* p, cudaStream_t stream) {
  return cudaFreeAsync(p, stream);
}

}  // namespace lw
