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

// edge: the exact-edge instantiation (Constant, Symmetric, Reflect;
// compiled wavelets).
cudaError_t launch_wrow_f32(int wi, int op, int p0, const WRowParams<float>& p,
                            int grid, int block, size_t smem, cudaStream_t stream, bool edge);
cudaError_t launch_wrow_f64(int wi, int op, int p0, const WRowParams<double>& p,
                            int grid, int block, size_t smem, cudaStream_t stream, bool edge);

// Two warps per row (float32 rows of 128 * p0 elements, p0 16 or 32; 128
// threads = two rows per CTA): levels compiled, 0 if none; launcher.
int wrow2_levels_f32(int wi, int op, int p0);
cudaError_t launch_wrow2_f32(int wi, int op, int p0, const WRowParams<float>& p, int grid,
                             size_t smem, cudaStream_t stream, bool edge);
// CTAs per SM the two-warp kernel's shared memory allows (grid sizing of
// the persistent launch).
int wrow2_resident_ctas(int p0);
// Whether contiguous float32 rows may use it (the "wrow_split" option).
bool wrow2_enabled();

// Windowed rows (rows longer than one warp holds): pairs per lane of the
// window (32 for float32, 16 for float64), levels compiled for (catalogue
// wavelet, transform), launchers.
template <typename T>
struct WTileParams;
int wtile_pairs(int elem_bytes);
int wtile_levels(int wi, int op, int elem_bytes);
// end_mask: the row length is a multiple of 2^levels but not of 2 * pairs
cudaError_t launch_wtile_f32(int wi, int op, bool end_mask, const WTileParams<float>& p, int grid,
                             size_t smem, cudaStream_t stream);
cudaError_t launch_wtile_f64(int wi, int op, bool end_mask, const WTileParams<double>& p,
                             int grid, size_t smem, cudaStream_t stream);
// Whether long contiguous rows may use it (the "row_windows" option).
bool wtile_enabled();
// Whether catalogue wavelets without compiled kernels may use the generic
// instantiations (the "generic_kernels" option).
bool generic_enabled();

}  // namespace lw
