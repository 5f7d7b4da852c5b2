// Host interface of the register-blocked fast path (lw_reg_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "lw_host.hpp"
#include "lw_types.hpp"

namespace lw {

template <typename T>
struct RegPassArgs {
  const DevProgram<T>* prog;  // resolved program for (wavelet, op, T)
  int wi;                     // catalogue index, -1 for user programs
  int op;
  int bc;
  int levels;                 // levels of this axis pass (>= 1)
  LineGeom g;
  const T* in;
  T* out;
  bool in_place;              // in and out overlap
};

struct RegStats {
  int launches = 0;
};

// One launch of kernel family `fam` (KernelFamily, lw_host.hpp).
inline void counted(RegStats* stats, int fam) {
  if (stats) stats->launches += 1;
  count_family(fam, 1);
}

// Runs one axis pass on the register path when it applies.  Returns 1 when
// launched, 0 when the pass is not eligible (the caller falls back to the
// general line kernel), a negative value on a CUDA failure.
template <typename T>
int plan_reg_pass(const RegPassArgs<T>& a, cudaStream_t stream, RegStats* stats);

// Whether strided float32 passes may use the TMA-staged kernel (the
// "tma_strided" option; on by default).
bool col_enabled();
// Whether it may pack two adjacent lines per lane (the "tma_packed" option).
bool col_packed();
// Whether short strided lines of a 3D view stack several outer slices in
// one staging window (the "tma_stacked" option).
bool col_stacked();
// Whether its tiles run in row-tile-major order (the "col_row_order"
// option).
bool col_row_order();
// Synchronises `stream`; returns 1 (and clears it) if a TMA-staged kernel
// gave up waiting for a staging copy since the last check, 0 if not, -1 if
// the check itself failed.
int check_col_errors(cudaStream_t stream);

}  // namespace lw
