/* CPU oracle for the lifting-scheme DWT of jcapriot/lifted -- see
 * lifted_oracle.h.  TEST INFRASTRUCTURE ONLY: loaded by tests/, the smoke
 * check and bench.py's CPU-baseline leg, never by the GPU library.
 *
 * Build: oracle/build_oracle.sh (gcc, -O2 -mfma -ffp-contract=off so that
 * every fused multiply-add in the restatement is an explicit fma() call and
 * nothing else is contracted). */
#include "lifted_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LO_K_GEN 0
#define LO_K_UNIT 1
#define LO_K_REPEAT 2
#define LO_K_SCALE 3
#define LO_EVENS 0
#define LO_ODDS 1
#define LO_TF_F 0
#define LO_TF_I 1
#define LO_TF_FA 2
#define LO_TF_IA 3
#define LO_BC_ZERO 0
#define LO_BC_CONSTANT 1
#define LO_BC_PERIODIC 2
#define LO_BC_SYMMETRIC 3
#define LO_BC_REFLECT 4
#define LO_MAX_TAPS 9
#define LO_MAX_STEPS 64

/* The catalogue table shared with the GPU library (generated from the
 * reference's src/lifted-wavelets.hpp; literals verbatim). */
#define LW_K_GEN LO_K_GEN
#define LW_K_UNIT LO_K_UNIT
#define LW_K_REPEAT LO_K_REPEAT
#define LW_K_SCALE LO_K_SCALE
#define LW_EVENS LO_EVENS
#define LW_ODDS LO_ODDS
#define LW_PM_ADD 0
#define LW_PM_SUB 1
#include "../lifted_b200/csrc/wavelet_catalogue.inc"

typedef struct {
  int kind, target, offset, ntaps, pm;
  long double c[LO_MAX_TAPS];
} lo_prog_row;

typedef struct {
  const char* name;
  uint32_t value, width, first, count;
} lo_cat_wavelet;

static const lo_prog_row LO_CAT_STEPS[] = {
#define LW_CATALOGUE_STEPS
#include "../lifted_b200/csrc/wavelet_catalogue.inc"
#undef LW_CATALOGUE_STEPS
};

static const lo_cat_wavelet LO_CAT_WAVELETS[] = {
#define LW_CATALOGUE_WAVELETS
#include "../lifted_b200/csrc/wavelet_catalogue.inc"
#undef LW_CATALOGUE_WAVELETS
};

static const lo_cat_wavelet* lo_find(uint32_t value) {
  size_t i;
  for (i = 0; i < sizeof(LO_CAT_WAVELETS) / sizeof(LO_CAT_WAVELETS[0]); ++i)
    if (LO_CAT_WAVELETS[i].value == value) return &LO_CAT_WAVELETS[i];
  return NULL;
}

size_t lo_wavelet_count(void) {
  return sizeof(LO_CAT_WAVELETS) / sizeof(LO_CAT_WAVELETS[0]);
}

uint32_t lo_wavelet_value(size_t index) {
  return index < lo_wavelet_count() ? LO_CAT_WAVELETS[index].value : 0xffffffffu;
}

size_t lo_wavelet_width(uint32_t wavelet) {
  const lo_cat_wavelet* w = lo_find(wavelet);
  return w ? w->width : (size_t)-1;
}

/* max_level (src/lifted-common.hpp:1099-1108). */
size_t lo_max_level(size_t width, size_t n) {
  size_t lvl = 0;
  if (width == 0) return 0;
  if (width == 1) return (size_t)-1;
  if (n < width - 1) return 0;
  while (n >= 2 * (width - 1)) {
    lvl += 1;
    n = (n + 1) / 2;
  }
  return lvl;
}

/* Boundary index maps (src/lifted-common.hpp:719-779).  Returns n for "skip
 * this tap" (Zero).  Periodic is the reference's i % n with i converted to an
 * unsigned 64-bit value, which wraps correctly only for power-of-two n.
 * Inputs on which the reference divides by zero (Periodic, n == 0) or loops
 * forever (Symmetric/Reflect with n == 0, Reflect with n == 1 and i outside
 * [0, 1)) set *err and return n. */
/* Which of the reference's two orderings of the adjoint back region to
 * restate: 1 (default) = the Across form, taken by every group of `lanes`
 * lines; 0 = the Along form, taken by the remaining lines. */
static int lo_fold_across = 1;
void lo_set_fold_order(int across) { lo_fold_across = across ? 1 : 0; }

static size_t lo_bc_index(int bc, ptrdiff_t i, size_t n, int* err) {
  ptrdiff_t io = i;
  switch (bc) {
    case LO_BC_ZERO:
      return (i < 0 || i >= (ptrdiff_t)n) ? n : (size_t)i;
    case LO_BC_CONSTANT:
      if (i < 0) return 0;
      if (i >= (ptrdiff_t)n) return n - 1;
      return (size_t)i;
    case LO_BC_PERIODIC:
      if (n == 0) { *err = 1; return n; }
      return ((size_t)i) % n;
    case LO_BC_SYMMETRIC:
      if (n == 0) { *err = 1; return n; }
      while (io >= (ptrdiff_t)n || io < 0) {
        if (io < 0) io = -(io + 1);
        else io = 2 * ((ptrdiff_t)n - 1) - (io - 1);
      }
      return (size_t)io;
    case LO_BC_REFLECT:
      if (n == 0 || (n == 1 && (i < 0 || i >= 1))) { *err = 1; return n; }
      while (io >= (ptrdiff_t)n || io < 0) {
        if (io < 0) io = -io;
        else io = 2 * ((ptrdiff_t)n - 1) - io;
      }
      return (size_t)io;
    default:
      *err = 1;
      return n;
  }
}

/* Loads the step rows of a catalogue wavelet or of a user program. */
static int lo_rows(uint32_t wavelet, const lo_user_step* up, size_t nup,
                   lo_prog_row* rows, size_t* n, size_t* width) {
  size_t k, t;
  if (up) {
    if (nup > LO_MAX_STEPS) return 1;
    for (k = 0; k < nup; ++k) {
      const lo_user_step* u = &up[k];
      if (u->kind > 3 || u->target > 1) return 1;
      if (u->kind == LO_K_SCALE && (u->ntaps < 1 || u->ntaps > 2)) return 1;
      if ((u->kind == LO_K_GEN || u->kind == LO_K_REPEAT) &&
          (u->ntaps < 1 || u->ntaps > LO_MAX_TAPS))
        return 1;
      memset(&rows[k], 0, sizeof(rows[k]));
      rows[k].kind = (int)u->kind;
      rows[k].target = (int)u->target;
      rows[k].offset = u->offset;
      rows[k].ntaps = (u->kind == LO_K_UNIT) ? 1 : (int)u->ntaps;
      rows[k].pm = (int)u->unit_sub;
      for (t = 0; t < LO_MAX_TAPS; ++t) rows[k].c[t] = (long double)u->coef[t];
    }
    *n = nup;
    *width = 0;
    return 0;
  } else {
    const lo_cat_wavelet* w = lo_find(wavelet);
    if (!w) return 1;
    for (k = 0; k < w->count; ++k) rows[k] = LO_CAT_STEPS[w->first + k];
    *n = w->count;
    *width = w->width;
    return 0;
  }
}

#define T float
#define SUF f32
#define FMA fmaf
#include "lifted_oracle_impl.h"
#undef T
#undef SUF
#undef FMA

#define T double
#define SUF f64
#define FMA fma
#include "lifted_oracle_impl.h"
#undef T
#undef SUF
#undef FMA
