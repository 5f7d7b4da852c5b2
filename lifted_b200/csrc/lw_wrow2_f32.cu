// Instantiations of the two-warp-per-row kernel (lw_wrow2_kernel.cuh).
#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_pdl.hpp"
#include "lw_wrow.hpp"
#include "lw_wrow2_kernel.cuh"

namespace lw {

namespace {

template <int WI, int OP, int P0, bool EDGE>
cudaError_t launch_one(const WRowParams<float>& p, int grid, size_t smem, cudaStream_t stream) {
  auto kern = wrow2_kernel<WI, OP, P0, EDGE>;
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

using Fn = cudaError_t (*)(const WRowParams<float>&, int, size_t, cudaStream_t);

template <int WI, int P0, bool EDGE>
Fn by_op(int op) {
  switch (op) {
    case 0: return launch_one<WI, 0, P0, EDGE>;
    case 1: return launch_one<WI, 1, P0, EDGE>;
    case 2: return launch_one<WI, 2, P0, EDGE>;
    default: return launch_one<WI, 3, P0, EDGE>;
  }
}

template <int P0, bool EDGE>
Fn by_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<2, P0, EDGE>(op);
    case 4: return by_op<4, P0, EDGE>(op);
    case 33: return by_op<33, P0, EDGE>(op);
    default: return nullptr;
  }
}

}  // namespace

int wrow2_levels_f32(int wi, int op, int p0) {
  if (wi != 2 && wi != 4 && wi != 33) return 0;
  if (p0 != 16 && p0 != 32) return 0;
  return reg_max_levels(wi, op, p0);
}

cudaError_t launch_wrow2_f32(int wi, int op, int p0, const WRowParams<float>& p, int grid,
                             size_t smem, cudaStream_t stream, bool edge) {
  Fn fn = nullptr;
  if (p0 == 16) fn = edge ? by_wavelet<16, true>(wi, op) : by_wavelet<16, false>(wi, op);
  if (p0 == 32) fn = edge ? by_wavelet<32, true>(wi, op) : by_wavelet<32, false>(wi, op);
  if (!fn) return cudaErrorInvalidValue;
  return fn(p, grid, smem, stream);
}

int wrow2_resident_ctas(int p0) {
  // shared memory bounds residency: two row slots, two buffers each
  const size_t smem = (size_t)4 * 128 * p0 * sizeof(float) + 256;
  const int per_sm = (int)((227 * 1024) / smem);
  return per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
}

}  // namespace lw
