// Launchers of the register-blocked kernel instantiations
// (lw_reg_inst_f32.cu, lw_reg_inst_f64.cu).
#pragma once

#include <cuda_runtime.h>

#include "lw_types.hpp"

namespace lw {

template <typename T>
struct RegParams;

template <typename T>
using RegFn = cudaError_t (*)(const RegParams<T>&, int, int, size_t,
                              cudaStream_t);

// Launcher for (catalogue wavelet, transform, strided mapping, tile mode,
// lines per lane, exact band edges of the non-Zero boundaries); nullptr
// when that combination is not compiled.
RegFn<float> pick_reg_f32(int wi, int op, bool strided, bool tile, int v, bool edge);
RegFn<double> pick_reg_f64(int wi, int op, bool strided, bool tile, int v, bool edge);

}  // namespace lw
