/* CPU oracle for the lifting-scheme DWT of jcapriot/lifted.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a scalar restatement, in plain C, of the
 * reference's algorithm for the hot path (steps, per-axis multi-level
 * drivers, separable and non-separable nD drivers).  It exists to check the
 * GPU library; only tests/, the smoke check and bench.py's CPU-baseline leg
 * may load it, and never as the thing measured or shipped.
 *
 * Parity of this restatement is pinned against the reference itself: the
 * tests compare it, bit for bit, with the reference's own sources compiled in
 * oracle/_ref (see build_ref.sh) on every catalogue wavelet, every boundary
 * condition, all four transforms and odd/even/short lengths.
 *
 * Arithmetic follows the reference exactly: every multiply-add of a lifting
 * tap is fused (one rounding), as Highway's MulAdd/NegMulAdd and GCC's
 * default contraction of the scalar edge loops make it; repeat steps sum
 * their taps before the single fused multiply-add; scale steps multiply.
 *
 * Return codes (shared with the GPU library's C ABI):
 *   0  ok
 *   1  invalid argument (bad enum value, axis out of range, ...)
 *   2  degenerate input on which the reference hangs, divides by zero or
 *      reads/writes out of bounds (see lo_bc_index and the fold loops).
 */
#ifndef LIFTED_ORACLE_H_
#define LIFTED_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One lifting step of a user-supplied program (the layout of lifted_step_t
 * in the GPU library's C ABI). */
typedef struct lo_user_step {
  uint32_t kind;     /* 0 generic, 1 unit, 2 repeat, 3 scale */
  uint32_t target;   /* 0 updates evens (s), 1 updates odds (d) */
  int32_t offset;
  uint32_t ntaps;    /* generic/repeat tap count; scale: 1 or 2 factors */
  uint32_t unit_sub; /* unit steps: 1 subtract, 0 add */
  uint32_t pad_;
  double coef[9];
} lo_user_step;

/* wavelet: catalogue enum value, used when prog == NULL.  prog/nprog/width:
 * a user step program (width only matters for level 0 = max level). */
int lo_sep_f32(uint32_t wavelet, const lo_user_step* prog, size_t nprog,
               size_t width, uint32_t tf, uint32_t bc, size_t ndim,
               const size_t* shape, const ptrdiff_t* sin,
               const ptrdiff_t* sout, size_t naxes, const size_t* axes,
               const size_t* levels, const float* in, float* out);
int lo_sep_f64(uint32_t wavelet, const lo_user_step* prog, size_t nprog,
               size_t width, uint32_t tf, uint32_t bc, size_t ndim,
               const size_t* shape, const ptrdiff_t* sin,
               const ptrdiff_t* sout, size_t naxes, const size_t* axes,
               const size_t* levels, const double* in, double* out);
int lo_nonsep_f32(uint32_t wavelet, const lo_user_step* prog, size_t nprog,
                  size_t width, uint32_t tf, uint32_t bc, size_t ndim,
                  const size_t* shape, const ptrdiff_t* sin,
                  const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                  size_t level, const float* in, float* out);
int lo_nonsep_f64(uint32_t wavelet, const lo_user_step* prog, size_t nprog,
                  size_t width, uint32_t tf, uint32_t bc, size_t ndim,
                  const size_t* shape, const ptrdiff_t* sin,
                  const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                  size_t level, const double* in, double* out);
/* FixedTransform::apply on pre-split bands (one level, no (de)interleave). */
int lo_fixed_apply_f32(uint32_t wavelet, const lo_user_step* prog,
                       size_t nprog, uint32_t tf, uint32_t bc, float* s,
                       float* d, size_t ns, size_t nd);
int lo_fixed_apply_f64(uint32_t wavelet, const lo_user_step* prog,
                       size_t nprog, uint32_t tf, uint32_t bc, double* s,
                       double* d, size_t ns, size_t nd);
/* Adjoint back-region ordering: 1 (default) restates the reference's Across
 * form (back fold, then the direct loop), 0 its Along form (direct loop,
 * then the back fold).  Only rounding differs between the two. */
void lo_set_fold_order(int across);
/* Catalogue queries. */
size_t lo_wavelet_count(void);
uint32_t lo_wavelet_value(size_t index);
size_t lo_wavelet_width(uint32_t wavelet); /* (size_t)-1 if unknown */
/* max_level(width, n); returns (size_t)-1 for width 1 (the reference never
 * returns there). */
size_t lo_max_level(size_t width, size_t n);

#ifdef __cplusplus
}
#endif
#endif
