// Instantiations of the windowed warp-per-row kernel (lw_wtile_kernel.cuh):
// float32 windows of 2048 samples (32 pairs per lane), float64 windows of
// 1024 (16 pairs per lane), for the compiled catalogue wavelets.
#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_pdl.hpp"
#include "lw_wrow.hpp"
#include "lw_wtile_kernel.cuh"

namespace lw {

namespace {

template <typename T, int WI, int OP, int P0, bool EM>
cudaError_t launch_one(const WTileParams<T>& p, int grid, size_t smem, cudaStream_t stream) {
  auto kern = wtile_kernel<T, WI, OP, P0, EM>;
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
  return launch_overlapped(kern, grid, 128, smem, stream, p);
}

template <typename T>
using Fn = cudaError_t (*)(const WTileParams<T>&, int, size_t, cudaStream_t);

template <typename T, int WI, int P0, bool EM>
Fn<T> by_op(int op) {
  switch (op) {
    case 0: return launch_one<T, WI, 0, P0, EM>;
    case 1: return launch_one<T, WI, 1, P0, EM>;
    case 2: return launch_one<T, WI, 2, P0, EM>;
    default: return launch_one<T, WI, 3, P0, EM>;
  }
}

template <typename T, int P0, bool EM>
Fn<T> by_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<T, 2, P0, EM>(op);
    case 4: return by_op<T, 4, P0, EM>(op);
    case 33: return by_op<T, 33, P0, EM>(op);
    case WI_GEN: return by_op<T, WI_GEN, P0, EM>(op);
    default: return nullptr;
  }
}

}  // namespace

int wtile_pairs(int elem_bytes) { return elem_bytes == 4 ? 32 : 16; }

int wtile_levels(int wi, int op, int elem_bytes) {
  // every catalogue wavelet: compiled ones directly, the others through the
  // generic instantiation
  if (wi < 0 || wi >= kNumCatalogue) return 0;
  return reg_max_levels(wi, op, wtile_pairs(elem_bytes));
}

cudaError_t launch_wtile_f32(int wi, int op, bool end_mask, const WTileParams<float>& p, int grid,
                             size_t smem, cudaStream_t stream) {
  Fn<float> fn = end_mask ? by_wavelet<float, 32, true>(wi, op) : by_wavelet<float, 32, false>(wi, op);
  if (!fn) return cudaErrorInvalidValue;
  return fn(p, grid, smem, stream);
}

cudaError_t launch_wtile_f64(int wi, int op, bool end_mask, const WTileParams<double>& p,
                             int grid, size_t smem, cudaStream_t stream) {
  Fn<double> fn =
      end_mask ? by_wavelet<double, 16, true>(wi, op) : by_wavelet<double, 16, false>(wi, op);
  if (!fn) return cudaErrorInvalidValue;
  return fn(p, grid, smem, stream);
}

}  // namespace lw
