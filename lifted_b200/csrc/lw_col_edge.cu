// Exact-edge instantiations of the TMA-staged strided kernel (Constant,
// Symmetric and Reflect boundaries; compiled wavelets, one line per lane).
#include "lw_col_inst.cuh"

namespace lw {

ColFn<float> pick_col_f32_edge(int wi, int op) { return colinst::edge_wavelet<float, 1>(wi, op); }
ColFn<double> pick_col_f64_edge(int wi, int op) {
  return colinst::edge_wavelet<double, 1>(wi, op);
}

}  // namespace lw
