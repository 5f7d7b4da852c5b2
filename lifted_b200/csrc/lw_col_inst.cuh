// Instantiation helpers of the TMA-staged strided kernel (lw_col_kernel.cuh),
// shared by the translation units that instantiate it (lw_col_f32.cu,
// lw_col_f64.cu, lw_col_edge.cu, lw_col_ldg.cu: split so that they compile
// in parallel).
#pragma once

#include <cuda_runtime.h>

#include "lw_col.hpp"
#include "lw_col_kernel.cuh"
#include "lw_launch.hpp"
#include "lw_pdl.hpp"

namespace lw {
namespace colinst {


template <typename T, int WI, int OP, int V, bool EM, bool EDGE, bool LDG = false>
cudaError_t launch_one(const ColParams<T>& p, int grid, size_t smem, cudaStream_t stream) {
  auto kern = col_kernel<T, WI, OP, V, EM, EDGE, LDG>;
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
  return launch_overlapped_kind(1, kern, grid, COL_THREADS, smem, stream, p);
}

template <typename T, int WI, int V, bool EM, bool EDGE = false, bool LDG = false>
ColFn<T> by_op(int op) {
  switch (op) {
    case 0: return launch_one<T, WI, 0, V, EM, EDGE, LDG>;
    case 1: return launch_one<T, WI, 1, V, EM, EDGE, LDG>;
    case 2: return launch_one<T, WI, 2, V, EM, EDGE, LDG>;
    default: return launch_one<T, WI, 3, V, EM, EDGE, LDG>;
  }
}

// The compiled wavelets with exact band edges (Constant, Symmetric,
// Reflect; whole chunks only).
template <typename T, int V>
ColFn<T> edge_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<T, 2, V, false, true>(op);
    case 4: return by_op<T, 4, V, false, true>(op);
    case 33: return by_op<T, 33, V, false, true>(op);
    default: return nullptr;
  }
}

template <typename T, int V, bool EM, bool LDG = false>
ColFn<T> by_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<T, 2, V, EM, false, LDG>(op);
    case 4: return by_op<T, 4, V, EM, false, LDG>(op);
    case 33: return by_op<T, 33, V, EM, false, LDG>(op);
    case WI_GEN: return by_op<T, WI_GEN, V, EM, false, LDG>(op);
    case WI_GENW:
      if constexpr (V == 1) return by_op<T, WI_GENW, V, EM, false, LDG>(op);
      else return nullptr;
    default: return nullptr;
  }
}


}  // namespace colinst
}  // namespace lw
