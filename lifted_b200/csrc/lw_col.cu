// Instantiations of the TMA-staged strided kernel (lw_col_kernel.cuh) for
// the compiled catalogue wavelets.
#include <cuda_runtime.h>

#include "lw_col.hpp"
#include "lw_col_kernel.cuh"
#include "lw_launch.hpp"
#include "lw_pdl.hpp"

namespace lw {
namespace {

template <typename T, int WI, int OP, int V, bool EM, bool EDGE>
cudaError_t launch_one(const ColParams<T>& p, int grid, size_t smem, cudaStream_t stream) {
  auto kern = col_kernel<T, WI, OP, V, EM, EDGE>;
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

template <typename T, int WI, int V, bool EM, bool EDGE = false>
ColFn<T> by_op(int op) {
  switch (op) {
    case 0: return launch_one<T, WI, 0, V, EM, EDGE>;
    case 1: return launch_one<T, WI, 1, V, EM, EDGE>;
    case 2: return launch_one<T, WI, 2, V, EM, EDGE>;
    default: return launch_one<T, WI, 3, V, EM, EDGE>;
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

template <typename T, int V, bool EM>
ColFn<T> by_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<T, 2, V, EM>(op);
    case 4: return by_op<T, 4, V, EM>(op);
    case 33: return by_op<T, 33, V, EM>(op);
    case WI_GEN: return by_op<T, WI_GEN, V, EM>(op);
    case WI_GENW:
      if constexpr (sizeof(T) == 4 && V == 1) return by_op<T, WI_GENW, V, EM>(op);
      else return nullptr;
    default: return nullptr;
  }
}

}  // namespace

// em: lines whose length is not a multiple of 32 (one line per lane only);
// edge: the exact-edge instantiation (non-Zero boundaries)
ColFn<float> pick_col_f32(int wi, int op, int v, bool em, bool edge) {
  if (edge) return (em || v != 1) ? nullptr : edge_wavelet<float, 1>(wi, op);
  if (em) return v == 1 ? by_wavelet<float, 1, true>(wi, op) : nullptr;
  return v == 2 ? by_wavelet<float, 2, false>(wi, op) : by_wavelet<float, 1, false>(wi, op);
}
ColFn<double> pick_col_f64(int wi, int op, bool em, bool edge) {
  if (edge) return em ? nullptr : edge_wavelet<double, 1>(wi, op);
  return em ? by_wavelet<double, 1, true>(wi, op) : by_wavelet<double, 1, false>(wi, op);
}

size_t col_smem_bytes(int hmax, int v, int elem_bytes) {
  return (size_t)COL_ROWS * COL_LANES * v * elem_bytes +
         (size_t)4 * hmax * COL_THREADS * v * elem_bytes + 16;
}

}  // namespace lw
