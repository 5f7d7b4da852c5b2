// Instantiations of the TMA-staged strided kernel (lw_col_kernel.cuh) for
// the compiled catalogue wavelets.
#include <cuda_runtime.h>

#include "lw_col.hpp"
#include "lw_col_kernel.cuh"
#include "lw_launch.hpp"

namespace lw {
namespace {

template <int WI, int OP, int V>
cudaError_t launch_one(const ColParams& p, int grid, size_t smem, cudaStream_t stream) {
  auto kern = col_kernel<WI, OP, V>;
  static bool configured[kMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!configured[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kMaxDynSmem);
    if (e != cudaSuccess) return e;
    configured[dev] = true;
  }
  kern<<<grid, COL_THREADS, smem, stream>>>(p);
  return cudaGetLastError();
}

template <int WI, int V>
ColFn by_op(int op) {
  switch (op) {
    case 0: return launch_one<WI, 0, V>;
    case 1: return launch_one<WI, 1, V>;
    case 2: return launch_one<WI, 2, V>;
    default: return launch_one<WI, 3, V>;
  }
}

template <int V>
ColFn by_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<2, V>(op);
    case 4: return by_op<4, V>(op);
    case 33: return by_op<33, V>(op);
    default: return nullptr;
  }
}

}  // namespace

ColFn pick_col(int wi, int op, int v) {
  return v == 2 ? by_wavelet<2>(wi, op) : by_wavelet<1>(wi, op);
}

size_t col_smem_bytes(int hmax, int v) {
  return (size_t)COL_ROWS * COL_LANES * v * sizeof(float) +
         (size_t)4 * hmax * COL_THREADS * v * sizeof(float) + 16;
}

}  // namespace lw
