// Instantiations of the register-blocked kernel (lw_reg_kernel.cuh) for double.
#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_pdl.hpp"
#include "lw_reg_inst.hpp"
#include "lw_reg_kernel.cuh"

namespace lw {
namespace {

constexpr int P0 = 8;

template <int WI, int OP, bool STRIDED, bool TILE, int V, bool EDGE>
cudaError_t launch_one(const RegParams<double>& p, int grid, int block,
                       size_t smem, cudaStream_t stream) {
  auto kern = reg_kernel<double, WI, OP, P0, STRIDED, TILE, V, EDGE>;
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

template <int WI, int OP, bool EDGE>
RegFn<double> by_mode(bool strided, bool tile, int v) {
  if (!strided) return tile ? nullptr : launch_one<WI, OP, false, false, 1, EDGE>;
  if (v != 1) return nullptr;
  return tile ? launch_one<WI, OP, true, true, 1, EDGE>
              : launch_one<WI, OP, true, false, 1, EDGE>;
}

template <int WI, bool EDGE>
RegFn<double> by_op(int op, bool strided, bool tile, int v) {
  switch (op) {
    case 0: return by_mode<WI, 0, EDGE>(strided, tile, v);
    case 1: return by_mode<WI, 1, EDGE>(strided, tile, v);
    case 2: return by_mode<WI, 2, EDGE>(strided, tile, v);
    default: return by_mode<WI, 3, EDGE>(strided, tile, v);
  }
}

}  // namespace

RegFn<double> pick_reg_f64(int wi, int op, bool strided, bool tile, int v, bool edge) {
  switch (wi) {
    case 2: return edge ? by_op<2, true>(op, strided, tile, v) : by_op<2, false>(op, strided, tile, v);
    case 4: return edge ? by_op<4, true>(op, strided, tile, v) : by_op<4, false>(op, strided, tile, v);
    case 33:
      return edge ? by_op<33, true>(op, strided, tile, v) : by_op<33, false>(op, strided, tile, v);
    default: return nullptr;
  }
}

}  // namespace lw
