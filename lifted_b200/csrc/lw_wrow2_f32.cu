// Instantiations of the two-warp-per-row kernel (lw_wrow2_kernel.cuh).
#include <cuda_runtime.h>

#include "lw_launch.hpp"
#include "lw_pdl.hpp"
#include "lw_wrow.hpp"
#include "lw_wrow2_kernel.cuh"

namespace lw {

namespace {

template <int WI, int OP, int P0, bool DS>
cudaError_t launch_one(const WRowParams<float>& p, int grid, size_t smem, cudaStream_t stream) {
  auto kern = DS ? wrow2d_kernel<WI, OP, P0> : wrow2_kernel<WI, OP, P0>;
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

template <int WI, int P0, bool DS>
Fn by_op(int op) {
  switch (op) {
    case 0: return launch_one<WI, 0, P0, DS>;
    case 1: return launch_one<WI, 1, P0, DS>;
    case 2: return launch_one<WI, 2, P0, DS>;
    default: return launch_one<WI, 3, P0, DS>;
  }
}

template <int P0, bool DS>
Fn by_wavelet(int wi, int op) {
  switch (wi) {
    case 2: return by_op<2, P0, DS>(op);
    case 4: return by_op<4, P0, DS>(op);
    case 33: return by_op<33, P0, DS>(op);
    default: return nullptr;
  }
}

template <bool DS>
Fn pick(int wi, int op, int p0) {
  return p0 == 16 ? by_wavelet<16, DS>(wi, op) : (p0 == 32 ? by_wavelet<32, DS>(wi, op) : nullptr);
}

}  // namespace

int wrow2_levels_f32(int wi, int op, int p0) {
  if (wi != 2 && wi != 4 && wi != 33) return 0;
  if (p0 != 16 && p0 != 32) return 0;
  return reg_max_levels(wi, op, p0);
}

cudaError_t launch_wrow2_f32(int wi, int op, int p0, const WRowParams<float>& p, int grid,
                             size_t smem, cudaStream_t stream) {
  Fn fn = wrow2_direct() ? pick<true>(wi, op, p0) : pick<false>(wi, op, p0);
  if (!fn) return cudaErrorInvalidValue;
  return fn(p, grid, smem, stream);
}

size_t wrow2_smem(int p0) {
  // two row slots; the staged form keeps two buffers per slot (input and
  // output staging, the next row's copy), the direct-store form one
  return (size_t)(wrow2_direct() ? 2 : 4) * 128 * p0 * sizeof(float);
}

int wrow2_resident_ctas(int wi, int op, int p0) {
  int per_sm = 0;
  const size_t smem = wrow2_smem(p0);
  auto occ = [&](auto kern) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kMaxDynSmem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = (int)((227 * 1024) / (smem + 256));
    }
  };
  // the residency of one instantiation stands for all (same shape of work)
  if (wrow2_direct()) occ(wrow2d_kernel<33, 0, 32>);
  else occ(wrow2_kernel<33, 0, 32>);
  (void)wi;
  (void)op;
  return per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
}

}  // namespace lw
