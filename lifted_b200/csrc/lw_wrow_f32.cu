// Instantiations of the warp-per-row kernel (lw_wrow_kernel.cuh) for float.
#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_pdl.hpp"
#include "lw_wrow.hpp"
#include "lw_wrow_kernel.cuh"

namespace lw {

// The exact-edge instantiations (lw_wrow_f32_edge.cu).
using WRowFnf32 = cudaError_t (*)(const WRowParams<float>&, int, int, size_t, cudaStream_t);
WRowFnf32 wrow_edge_f32(int wi, int op, int p0);

namespace {

template <int WI, int OP, int P0, bool EDGE>
cudaError_t launch_one(const WRowParams<float>& p, int grid, int block,
                       size_t smem, cudaStream_t stream) {
  auto kern = wrow_kernel<float, WI, OP, P0, EDGE>;
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

using Fn = cudaError_t (*)(const WRowParams<float>&, int, int, size_t, cudaStream_t);

template <int WI, int P0, bool EDGE = false>
Fn by_op(int op) {
  switch (op) {
    case 0: return launch_one<WI, 0, P0, EDGE>;
    case 1: return launch_one<WI, 1, P0, EDGE>;
    case 2: return launch_one<WI, 2, P0, EDGE>;
    default: return launch_one<WI, 3, P0, EDGE>;
  }
}

template <int P0>
Fn by_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<2, P0>(op);
    case 4: return by_op<4, P0>(op);
    case 33: return by_op<33, P0>(op);
    case WI_GEN: return by_op<WI_GEN, P0>(op);
    default: return nullptr;
  }
}


}  // namespace

int wrow_levels_f32(int wi, int op, int p0) {
  switch (p0) {
    case 8: return (wi == 2 || wi == 4 || wi == 33) ? wrow_max_levels(wi, op, 8) : 0;
    case 16: return (wi == 2 || wi == 4 || wi == 33) ? wrow_max_levels(wi, op, 16) : 0;
    case 32: return (wi == 2 || wi == 4 || wi == 33) ? wrow_max_levels(wi, op, 32) : 0;
    case 64: return (wi == 2 || wi == 4 || wi == 33) ? wrow_max_levels(wi, op, 64) : 0;
    default: return 0;
  }
}

cudaError_t launch_wrow_f32(int wi, int op, int p0, const WRowParams<float>& p,
                            int grid, int block, size_t smem,
                            cudaStream_t stream, bool edge) {
  Fn fn = nullptr;
  switch (p0) {
    case 8: fn = edge ? wrow_edge_f32(wi, op, 8) : by_wavelet<8>(wi, op); break;
    case 16: fn = edge ? wrow_edge_f32(wi, op, 16) : by_wavelet<16>(wi, op); break;
    case 32: fn = edge ? wrow_edge_f32(wi, op, 32) : by_wavelet<32>(wi, op); break;
    case 64: fn = edge ? wrow_edge_f32(wi, op, 64) : by_wavelet<64>(wi, op); break;
    default: break;
  }
  if (!fn) return cudaErrorInvalidValue;
  return fn(p, grid, block, smem, stream);
}

}  // namespace lw
