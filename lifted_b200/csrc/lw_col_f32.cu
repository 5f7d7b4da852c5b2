// Instantiations of the TMA-staged strided kernel for float32, Zero
// boundary (compiled wavelets and the generic instantiations).
#include "lw_col_inst.cuh"

namespace lw {

ColFn<float> pick_col_f32_zero(int wi, int op, int v, bool em) {
  using namespace colinst;
  if (em) return v == 1 ? by_wavelet<float, 1, true>(wi, op) : nullptr;
  return v == 2 ? by_wavelet<float, 2, false>(wi, op) : by_wavelet<float, 1, false>(wi, op);
}

}  // namespace lw
