// Instantiations of the TMA-staged strided kernel for float64, Zero
// boundary (compiled wavelets and the generic instantiation).
#include "lw_col_inst.cuh"

namespace lw {

ColFn<double> pick_col_f64_zero(int wi, int op, bool em) {
  using namespace colinst;
  return em ? by_wavelet<double, 1, true>(wi, op) : by_wavelet<double, 1, false>(wi, op);
}

}  // namespace lw
