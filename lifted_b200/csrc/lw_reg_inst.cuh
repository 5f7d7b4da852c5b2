// Instantiation helpers of the register-blocked kernel (lw_reg_kernel.cuh),
// shared by its instantiation units (float32 and float64, Zero and
// exact-edge forms in separate units so that they compile in parallel).
#pragma once

#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_pdl.hpp"
#include "lw_reg_inst.hpp"
#include "lw_reg_kernel.cuh"

namespace lw {
namespace reginst {

template <typename T, int WI, int OP, bool STRIDED, bool TILE, int V, bool EDGE>
cudaError_t launch_one(const RegParams<T>& p, int grid, int block,
                       size_t smem, cudaStream_t stream) {
  auto kern = reg_kernel<T, WI, OP, (sizeof(T) == 4 ? 16 : 8), STRIDED, TILE, V, EDGE>;
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
  return launch_overlapped(kern, grid, block, smem, stream, p);
}

template <typename T, int WI, int OP, bool EDGE>
RegFn<T> by_mode(bool strided, bool tile, int v) {
  if (!strided) return tile ? nullptr : launch_one<T, WI, OP, false, false, 1, EDGE>;
  // two lines per lane: float32 only
  if constexpr (sizeof(T) == 4) {
    if (v == 2) return tile ? launch_one<T, WI, OP, true, true, 2, EDGE>
                            : launch_one<T, WI, OP, true, false, 2, EDGE>;
  }
  if (v != 1) return nullptr;
  return tile ? launch_one<T, WI, OP, true, true, 1, EDGE>
              : launch_one<T, WI, OP, true, false, 1, EDGE>;
}

template <typename T, int WI, bool EDGE>
RegFn<T> by_op(int op, bool strided, bool tile, int v) {
  switch (op) {
    case 0: return by_mode<T, WI, 0, EDGE>(strided, tile, v);
    case 1: return by_mode<T, WI, 1, EDGE>(strided, tile, v);
    case 2: return by_mode<T, WI, 2, EDGE>(strided, tile, v);
    default: return by_mode<T, WI, 3, EDGE>(strided, tile, v);
  }
}

}  // namespace reginst
}  // namespace lw
