// Host interface of the warp-per-row kernel (lw_wrow_f32.cu, lw_wrow_f64.cu).
#pragma once

#include <cuda_runtime.h>

#include "lw_types.hpp"

namespace lw {

template <typename T>
struct WRowParams;

// Levels one warp can run in registers for (catalogue wavelet, transform,
// pairs per lane); 0 when that combination is not compiled.
int wrow_levels_f32(int wi, int op, int p0);
int wrow_levels_f64(int wi, int op, int p0);

cudaError_t launch_wrow_f32(int wi, int op, int p0, const WRowParams<float>& p,
                            int grid, int block, size_t smem, cudaStream_t stream);
cudaError_t launch_wrow_f64(int wi, int op, int p0, const WRowParams<double>& p,
                            int grid, int block, size_t smem, cudaStream_t stream);

}  // namespace lw
