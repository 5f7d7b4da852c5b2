// Types shared by the host planner and the CUDA kernels of the B200 lifting
// DWT.  A wavelet's step program is resolved on the host for one element
// type and one transform (src/lifted-common.hpp:798-996 hold the reference's
// compile-time equivalents) and handed to the kernels by value, already in
// execution order.
#pragma once

#include <cstddef>
#include <cstdint>

namespace lw {

enum StepKind : int32_t { K_GEN = 0, K_UNIT = 1, K_REPEAT = 2, K_SCALE = 3 };
enum Boundary : int32_t {
  BC_ZERO = 0,
  BC_CONSTANT = 1,
  BC_PERIODIC = 2,
  BC_SYMMETRIC = 3,
  BC_REFLECT = 4
};
enum TransformOp : int32_t { TF_F = 0, TF_I = 1, TF_FA = 2, TF_IA = 3 };

constexpr int MAX_TAPS = 9;
constexpr int MAX_STEPS = 32;
constexpr int MAX_NDIM = 16;
constexpr int MAX_LEVELS = 63;

// One lifting step resolved for one transform.
//   y_is_d   the updated band is d (x = s) when 1, s (x = d) when 0
//   sub      the update subtracts (ISub, or a reversed unit step)
//   off      offset of the first tap used by the direct loops
//            (OffsetData::offset for Forward/Inverse, offset_r for the
//            adjoints, src/lifted-common.hpp:810-821)
//   fold_off the step's own offset, where the adjoint front fold starts
//   nf, nb   n_front/n_back (or n_front_r/n_back_r)
//   c        tap coefficients as used (vals, or reversed vals_r for the
//            adjoints); repeat steps keep their single value in c[0]
//   sm, dm   scale multipliers of s and d for this transform (Q8)
template <typename T>
struct DevStep {
  int32_t kind;
  int32_t y_is_d;
  int32_t sub;
  int32_t ntaps;
  int32_t off;
  int32_t fold_off;
  int32_t nf;
  int32_t nb;
  int32_t shape;   // index in the generic kernels' step-shape table (-1: none)
  int32_t pad_;
  T c[MAX_TAPS];
  T sm;
  T dm;
};

// A step program in execution order (reversed for Inverse/ForwardAdjoint,
// src/lifted-drivers-inl.hpp:51-63).
template <typename T>
struct DevProgram {
  int32_t nsteps;
  int32_t normal;      // Forward or Inverse (not an adjoint)
  int32_t fwd_driver;  // forward-stepping driver: Forward, InverseAdjoint
  int32_t across;      // adjoint back region: 1 fold first (Across form),
                       // 0 direct loop first (Along form)
  DevStep<T> st[MAX_STEPS];
};

// The lines of one axis pass: every line along `axis` of an nD array.
// Other dims are listed fastest-varying first (smallest |stride_out|), so
// that consecutive line indices are adjacent in memory where possible.
struct LineGeom {
  int64_t n;       // length along the axis
  int64_t sin;     // axis stride of the source (elements)
  int64_t sout;    // axis stride of the destination
  int64_t nlines;  // product of the other dims
  int32_t nother;
  int32_t pad_;
  int64_t oshape[MAX_NDIM];
  int64_t oin[MAX_NDIM];
  int64_t oout[MAX_NDIM];
};

// Kernel parameters of the general line kernel.
template <typename T>
struct LineParams {
  const T* in;
  T* out;
  LineGeom g;
  int32_t levels;
  int32_t bc;
  int32_t W;          // lines per CTA
  int32_t use_smem;   // 1: buffers in dynamic shared memory
  int32_t zfast;      // 1: Zero boundary, direct step code (zero_step)
  int32_t pad_;
  int64_t pitch;      // elements per line in buffer A
  int64_t pitch_b;    // elements per line in buffer B
  T* scratch;         // global buffers when use_smem == 0
  int64_t nlines_per_cta_stride;  // grid stride in lines
  DevProgram<T> prog;
};

}  // namespace lw
