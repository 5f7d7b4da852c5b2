// Plain-load instantiations of the strided kernel (lw_col_kernel.cuh, LDG):
// lines whose stride, line count or base TMA cannot take; Zero boundary,
// one line per lane, end-masked (any line length).
#include "lw_col_inst.cuh"

namespace lw {

ColFn<float> pick_col_ldg_f32(int wi, int op) {
  return colinst::by_wavelet<float, 1, true, true>(wi, op);
}
ColFn<double> pick_col_ldg_f64(int wi, int op) {
  return colinst::by_wavelet<double, 1, true, true>(wi, op);
}

}  // namespace lw
