// Instantiations of the register-blocked kernel (lw_reg_kernel.cuh) for
// float, Zero boundary; the exact-edge forms are in lw_reg_inst_f32_edge.cu.
#include "lw_reg_inst.cuh"

namespace lw {

RegFn<float> pick_reg_f32_edge(int wi, int op, bool strided, bool tile, int v);

RegFn<float> pick_reg_f32(int wi, int op, bool strided, bool tile, int v, bool edge) {
  if (edge) return pick_reg_f32_edge(wi, op, strided, tile, v);
  using namespace reginst;
  switch (wi) {
    case 2: return by_op<float, 2, false>(op, strided, tile, v);
    case 4: return by_op<float, 4, false>(op, strided, tile, v);
    case 33: return by_op<float, 33, false>(op, strided, tile, v);
    default: return nullptr;
  }
}

}  // namespace lw
