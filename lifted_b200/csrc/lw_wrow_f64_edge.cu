// Exact-edge instantiations (Constant, Symmetric, Reflect) of the
// warp-per-row kernel (lw_wrow_kernel.cuh) for double.
#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_pdl.hpp"
#include "lw_wrow.hpp"
#include "lw_wrow_kernel.cuh"

namespace lw {

// The exact-edge instantiations (lw_wrow_f64_edge.cu).
using WRowFnf64 = cudaError_t (*)(const WRowParams<double>&, int, int, size_t, cudaStream_t);
WRowFnf64 wrow_edge_f64(int wi, int op, int p0);

namespace {

template <int WI, int OP, int P0, bool EDGE>
cudaError_t launch_one(const WRowParams<double>& p, int grid, int block,
                       size_t smem, cudaStream_t stream) {
  auto kern = wrow_kernel<double, WI, OP, P0, EDGE>;
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

using Fn = cudaError_t (*)(const WRowParams<double>&, int, int, size_t, cudaStream_t);

template <int WI, int P0, bool EDGE = false>
Fn by_op(int op) {
  switch (op) {
    case 0: return launch_one<WI, 0, P0, EDGE>;
    case 1: return launch_one<WI, 1, P0, EDGE>;
    case 2: return launch_one<WI, 2, P0, EDGE>;
    default: return launch_one<WI, 3, P0, EDGE>;
  }
}

// The exact-edge instantiations (Constant, Symmetric, Reflect) of the
// compiled wavelets.
template <int P0>
Fn edge_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<2, P0, true>(op);
    case 4: return by_op<4, P0, true>(op);
    case 33: return by_op<33, P0, true>(op);
    default: return nullptr;
  }
}

}  // namespace

WRowFnf64 wrow_edge_f64(int wi, int op, int p0) {
  switch (p0) {
    case 8: return edge_wavelet<8>(wi, op);
    case 16: return edge_wavelet<16>(wi, op);
    case 32: return edge_wavelet<32>(wi, op);
    default: return nullptr;
  }
}

}  // namespace lw
