// Launcher selection of the TMA-staged strided kernel (lw_col_kernel.cuh);
// the instantiations live in lw_col_f32.cu, lw_col_f64.cu and
// lw_col_edge.cu.
#include <cuda_runtime.h>

#include "lw_col.hpp"
#include "lw_col_kernel.cuh"

namespace lw {

ColFn<float> pick_col_f32_zero(int wi, int op, int v, bool em);
ColFn<double> pick_col_f64_zero(int wi, int op, bool em);
ColFn<float> pick_col_f32_edge(int wi, int op);
ColFn<double> pick_col_f64_edge(int wi, int op);

// em: lines whose length is not a multiple of 32 (one line per lane only);
// edge: the exact-edge instantiation (non-Zero boundaries)
ColFn<float> pick_col_f32(int wi, int op, int v, bool em, bool edge) {
  if (edge) return (em || v != 1) ? nullptr : pick_col_f32_edge(wi, op);
  return pick_col_f32_zero(wi, op, v, em);
}
ColFn<double> pick_col_f64(int wi, int op, bool em, bool edge) {
  if (edge) return em ? nullptr : pick_col_f64_edge(wi, op);
  return pick_col_f64_zero(wi, op, em);
}

size_t col_smem_bytes(int hmax, int v, int elem_bytes, int mb_bufs) {
  return (size_t)COL_ROWS * COL_LANES * v * elem_bytes +
         (size_t)2 * mb_bufs * hmax * COL_THREADS * v * elem_bytes + 16;
}

}  // namespace lw
