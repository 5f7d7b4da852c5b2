// Exact-edge instantiations (Constant, Symmetric, Reflect) of the
// register-blocked kernel for float.
#include "lw_reg_inst.cuh"

namespace lw {

RegFn<float> pick_reg_f32_edge(int wi, int op, bool strided, bool tile, int v) {
  using namespace reginst;
  switch (wi) {
    case 2: return by_op<float, 2, true>(op, strided, tile, v);
    case 4: return by_op<float, 4, true>(op, strided, tile, v);
    case 33: return by_op<float, 33, true>(op, strided, tile, v);
    default: return nullptr;
  }
}

}  // namespace lw
