/* Type-generic body of the CPU oracle; included by lifted_oracle.c once per
 * element type with T (float/double), SUF (f32/f64) and FMA (fmaf/fma)
 * defined.  TEST INFRASTRUCTURE ONLY (see lifted_oracle.h).
 *
 * Each function names the reference code it restates (paths relative to the
 * jcapriot/lifted tree). */

#define LO_CAT2(a, b) a##_##b
#define LO_CAT(a, b) LO_CAT2(a, b)
#define LO_FN(name) LO_CAT(name, SUF)

/* One resolved step for element type T: the coefficient casts of
 * src/lifted-common.hpp:824-964 (vals, reversed vals_r, repeat val, scale
 * s_mul/s_div/d_div/d_mul). */
typedef struct {
  int kind, target, offset, ntaps, pm;
  T vals[LO_MAX_TAPS], vals_r[LO_MAX_TAPS], val;
  T s_mul, s_div, d_div, d_mul;
} LO_FN(lo_step);

static void LO_FN(resolve)(const lo_prog_row* r, LO_FN(lo_step) * st) {
  int k;
  memset(st, 0, sizeof(*st));
  st->kind = r->kind;
  st->target = r->target;
  st->offset = r->offset;
  st->ntaps = r->ntaps;
  st->pm = r->pm;
  if (r->kind == LO_K_GEN) {
    for (k = 0; k < r->ntaps; ++k) st->vals[k] = (T)r->c[k];
    for (k = 0; k < r->ntaps; ++k) st->vals_r[k] = st->vals[r->ntaps - 1 - k];
  } else if (r->kind == LO_K_REPEAT) {
    st->val = (T)r->c[0];
  } else if (r->kind == LO_K_SCALE) {
    long double a = r->c[0];
    long double b = (r->ntaps == 2) ? r->c[1] : r->c[0];
    st->s_mul = (T)a;
    st->s_div = (T)(1.0L / a);
    st->d_div = (T)b;
    st->d_mul = (T)(1.0L / b);
  }
}

/* y op= v * x with one rounding (IAdd/ISub::fused_iop,
 * src/lifted-steps-inl.hpp:50-53,69-72). */
static inline T LO_FN(fop)(int sub, T v, T x, T y) {
  return sub ? FMA(-v, x, y) : FMA(v, x, y);
}

/* Generic / repeat inner product at y-index i with the boundary map bc over
 * an x band of length nx (ip::inner_product, scalar BC overloads,
 * src/lifted-steps-inl.hpp:213-255; the interior overloads :87-122 give the
 * same result whenever every tap is in range, so one function serves both). */
static T LO_FN(ip_bc)(const LO_FN(lo_step) * st, int sub, int adj, int bc,
                      T y, ptrdiff_t off, const T* x, ptrdiff_t i, size_t nx,
                      int* err) {
  int k;
  ptrdiff_t io = i + off;
  if (st->kind == LO_K_GEN) {
    const T* vs = adj ? st->vals_r : st->vals;
    for (k = 0; k < st->ntaps; ++k) {
      size_t ib = lo_bc_index(bc, io + k, nx, err);
      if (ib < nx) y = LO_FN(fop)(sub, vs[k], x[ib], y);
    }
  } else { /* repeat: sum the taps first, then one fused multiply-add */
    size_t ib = lo_bc_index(bc, io, nx, err);
    T x0 = (ib < nx) ? x[ib] : (T)0;
    for (k = 1; k < st->ntaps; ++k) {
      ib = lo_bc_index(bc, io + k, nx, err);
      if (ib < nx) x0 += x[ib];
    }
    y = LO_FN(fop)(sub, st->val, x0, y);
  }
  return y;
}

/* ip::inner_product_safe (src/lifted-steps-inl.hpp:296-328): taps starting
 * at x-index j, dropped when outside [0, nx). */
static T LO_FN(ip_safe)(const LO_FN(lo_step) * st, int sub, T y,
                        const T* x, ptrdiff_t j, size_t nx) {
  int k;
  if (st->kind == LO_K_GEN) {
    const T* vs = st->vals_r;
    for (k = 0; k < st->ntaps; ++k) {
      ptrdiff_t ii = j + k;
      if (ii >= 0 && ii < (ptrdiff_t)nx) y = LO_FN(fop)(sub, vs[k], x[ii], y);
    }
  } else {
    T x0 = (j >= 0 && j < (ptrdiff_t)nx) ? x[j] : (T)0;
    for (k = 1; k < st->ntaps; ++k) {
      ptrdiff_t ii = j + k;
      if (ii >= 0 && ii < (ptrdiff_t)nx) x0 += x[ii];
    }
    y = LO_FN(fop)(sub, st->val, x0, y);
  }
  return y;
}

/* One step on split bands s (ns) and d (nd), transform tf, boundary bc:
 * Step<...>::operator() for Along (src/lifted-steps-inl.hpp:383-498 generic,
 * 632-751 unit, 897-1009 repeat, 1137-1176 scale). */
static void LO_FN(step)(const LO_FN(lo_step) * st, int tf, int bc, T* s, T* d,
                        size_t ns, size_t nd, int* err) {
  size_t i;
  if (st->kind == LO_K_SCALE) {
    int fwd = (tf == LO_TF_F || tf == LO_TF_FA);
    T dm = fwd ? st->d_mul : st->d_div;
    T sm = fwd ? st->s_mul : st->s_div;
    for (i = 0; i < nd; ++i) d[i] *= dm;
    for (i = 0; i < ns; ++i) s[i] *= sm;
    return;
  }
  {
    const int normal = (tf == LO_TF_F || tf == LO_TF_I);
    const int target = normal ? LO_ODDS : LO_EVENS;
    const ptrdiff_t N = st->ntaps;
    const ptrdiff_t offset = st->offset;
    /* OffsetData (src/lifted-common.hpp:798-822) */
    const ptrdiff_t maxo = N - 1 + offset;
    const size_t n_front = offset < 0 ? (size_t)(-offset) : 0;
    const size_t n_back = maxo < 0 ? 0 : (size_t)maxo;
    const ptrdiff_t offset_r = -maxo;
    const ptrdiff_t maxo_r = N - 1 + offset_r;
    const size_t n_front_r = offset_r < 0 ? (size_t)(-offset_r) : 0;
    const size_t n_back_r = maxo_r < 0 ? 0 : (size_t)maxo_r;
    const size_t nf = normal ? n_front : n_front_r;
    const size_t nb = normal ? n_back : n_back_r;
    const ptrdiff_t off = normal ? offset : offset_r;
    const int same = (st->target == target);
    const size_t nx = same ? ns : nd;
    const T* x = same ? s : d;
    const size_t ny = same ? nd : ns;
    T* y = same ? d : s;
    const size_t n1 = nf < ny ? nf : ny;
    const size_t n2 = nd > nb ? nd - nb : 0;
    int sub;
    ptrdiff_t ii, j;
    if (st->kind == LO_K_UNIT) {
      /* unit_op_from_tf_t (src/lifted-steps-inl.hpp:623-626) */
      int fwdtf = (tf == LO_TF_F || tf == LO_TF_FA);
      sub = fwdtf ? st->pm : !st->pm;
    } else {
      sub = (tf == LO_TF_I || tf == LO_TF_IA); /* op_from_tf (:75-77) */
    }

    if (st->kind == LO_K_UNIT) {
      if (!normal) { /* front fold (:659-668) */
        for (ii = offset, j = 0; ii < 0 && j < (ptrdiff_t)nx; ++ii, ++j) {
          size_t io = lo_bc_index(bc, ii, ny, err);
          if (io != ny && (ptrdiff_t)io != ii) {
            if (io > ny) { *err = 1; continue; }
            y[io] = sub ? y[io] - x[j] : y[io] + x[j];
          }
        }
      }
      for (ii = 0; ii < (ptrdiff_t)n1; ++ii) {
        size_t ib = lo_bc_index(normal ? bc : LO_BC_ZERO, ii + off, nx, err);
        if (ib < nx) y[ii] = sub ? y[ii] - x[ib] : y[ii] + x[ib];
      }
      for (ii = (ptrdiff_t)n1; ii < (ptrdiff_t)n2; ++ii)
        y[ii] = sub ? y[ii] - x[ii + off] : y[ii] + x[ii + off];
      {
        /* Adjoint back region: the Along form runs the direct loop and then
         * the back fold (:715-735); the Across form runs the fold first
         * (:837-864).  lo_fold_across selects which one to restate. */
        int pass;
        for (pass = 0; pass < 2; ++pass) {
          int do_fold = (!normal) && (pass == (lo_fold_across ? 0 : 1));
          int do_direct = (pass == (lo_fold_across ? 1 : 0));
          if (do_direct) {
            for (ii = (ptrdiff_t)n2; ii < (ptrdiff_t)ny; ++ii) {
              size_t ib = lo_bc_index(normal ? bc : LO_BC_ZERO, ii + off, nx, err);
              if (ib < nx) y[ii] = sub ? y[ii] - x[ib] : y[ii] + x[ib];
            }
          }
          if (do_fold) {
            for (ii = (ptrdiff_t)nd, j = (ptrdiff_t)nd + off;
                 ii < (ptrdiff_t)nx - off; ++ii, ++j) {
              size_t io = lo_bc_index(bc, ii, ny, err);
              if (io != ny && (ptrdiff_t)io != ii) {
                if (io > ny || j < 0 || j >= (ptrdiff_t)nx) { *err = 1; continue; }
                y[io] = sub ? y[io] - x[j] : y[io] + x[j];
              }
            }
          }
        }
      }
      return;
    }

    /* generic and repeat */
    if (!normal) { /* front fold (:416-430, :925-939) */
      for (ii = offset, j = 1 - N; ii < 0; ++ii, ++j) {
        size_t io = lo_bc_index(bc, ii, ny, err);
        if (io != ny && (ptrdiff_t)io != ii) {
          if (io > ny) { *err = 1; continue; }
          y[io] = LO_FN(ip_safe)(st, sub, y[io], x, j, nx);
        }
      }
    }
    {
      int ebc = normal ? bc : LO_BC_ZERO;
      for (ii = 0; ii < (ptrdiff_t)n1; ++ii)
        y[ii] = LO_FN(ip_bc)(st, sub, !normal, ebc, y[ii], off, x, ii, nx, err);
      for (ii = (ptrdiff_t)n1; ii < (ptrdiff_t)n2; ++ii)
        y[ii] = LO_FN(ip_bc)(st, sub, !normal, LO_BC_ZERO, y[ii], off, x, ii,
                             nx, err);
      /* Adjoint back region: Along runs the direct loop, then the back fold
       * (:466-484, :977-995); Across runs the fold first (:576-598,
       * :1087-1109). */
      int pass;
      for (pass = 0; pass < 2; ++pass) {
        int do_fold = (!normal) && (pass == (lo_fold_across ? 0 : 1));
        int do_direct = (pass == (lo_fold_across ? 1 : 0));
        if (do_direct)
          for (ii = (ptrdiff_t)n2; ii < (ptrdiff_t)ny; ++ii)
            y[ii] = LO_FN(ip_bc)(st, sub, !normal, ebc, y[ii], off, x, ii, nx, err);
        if (do_fold) {
          for (ii = (ptrdiff_t)nd, j = (ptrdiff_t)nd + off;
               ii < (ptrdiff_t)nx - off; ++ii, ++j) {
            size_t io = lo_bc_index(bc, ii, ny, err);
            if (io != ny && (ptrdiff_t)io != ii) {
              if (io > ny) { *err = 1; continue; }
              y[io] = LO_FN(ip_safe)(st, sub, y[io], x, j, nx);
            }
          }
        }
      }
    }
  }
}

/* FixedTransform<W>::apply (src/lifted-drivers-inl.hpp:51-63): steps in
 * order for Forward/InverseAdjoint, reversed for Inverse/ForwardAdjoint. */
static void LO_FN(fixed)(const LO_FN(lo_step) * prog, size_t np, int tf,
                         int bc, T* s, T* d, size_t ns, size_t nd, int* err) {
  size_t k;
  int fwd_loop = (tf == LO_TF_F || tf == LO_TF_IA);
  for (k = 0; k < np; ++k) {
    size_t idx = fwd_loop ? k : np - 1 - k;
    LO_FN(step)(&prog[idx], tf, bc, s, d, ns, nd, err);
  }
}

/* Multi-level 1D driver on one line: src (stride sstr) -> dst (stride dstr).
 * Forward-stepping form (src/lifted-drivers-inl.hpp:75-142) for Forward and
 * InverseAdjoint, reverse-stepping form (:182-274) for Inverse and
 * ForwardAdjoint.  levels == 0 leaves dst untouched (:87, :194). */
static void LO_FN(line)(const LO_FN(lo_step) * prog, size_t np, int tf,
                        int bc, const T* src, ptrdiff_t sstr, T* dst,
                        ptrdiff_t dstr, size_t n, size_t levels, T* w0, T* w1,
                        int* err) {
  size_t i, lvl;
  int fwd_loop = (tf == LO_TF_F || tf == LO_TF_IA);
  if (levels == 0) return;
  if (fwd_loop) {
    size_t m = n;
    /* deinterleave the input line (deinterleave_input, ops :317-335) */
    for (i = 0; i < n; ++i) w0[i] = src[(ptrdiff_t)i * sstr];
    for (lvl = 0; lvl < levels; ++lvl) {
      size_t nd = m / 2, ns = m - nd;
      for (i = 0; i < nd; ++i) {
        w1[i] = w0[2 * i];
        w1[ns + i] = w0[2 * i + 1];
      }
      if (ns > nd) w1[ns - 1] = w0[m - 1];
      LO_FN(fixed)(prog, np, tf, bc, w1, w1 + ns, ns, nd, err);
      for (i = 0; i < nd; ++i) dst[(ptrdiff_t)(ns + i) * dstr] = w1[ns + i];
      for (i = 0; i < ns; ++i) w0[i] = w1[i];
      m = ns;
    }
    for (i = 0; i < m; ++i) dst[(ptrdiff_t)i * dstr] = w0[i];
  } else {
    size_t ns_l[64], nd_l[64];
    size_t m = n, ns, nd;
    for (lvl = 0; lvl < levels; ++lvl) {
      nd_l[lvl] = m / 2;
      ns_l[lvl] = m - m / 2;
      m = ns_l[lvl];
    }
    /* w0 holds the whole input line; w1 the working s|d pair */
    for (i = 0; i < n; ++i) w0[i] = src[(ptrdiff_t)i * sstr];
    ns = ns_l[levels - 1];
    for (i = 0; i < ns; ++i) w1[i] = w0[i];
    for (lvl = levels; lvl-- > 0;) {
      ns = ns_l[lvl];
      nd = nd_l[lvl];
      for (i = 0; i < nd; ++i) w1[ns + i] = w0[ns + i];
      LO_FN(fixed)(prog, np, tf, bc, w1, w1 + ns, ns, nd, err);
      /* interleave s|d into the next level's s (ops :159-188) */
      {
        T* tmp = w1 + 2 * n + 2; /* scratch past the working pair */
        for (i = 0; i < ns + nd; ++i) tmp[i] = w1[i];
        for (i = 0; i < nd; ++i) {
          w1[2 * i] = tmp[i];
          w1[2 * i + 1] = tmp[ns + i];
        }
        if (ns > nd) w1[ns + nd - 1] = tmp[ns - 1];
      }
    }
    for (i = 0; i < n; ++i) dst[(ptrdiff_t)i * dstr] = w1[i];
  }
}

static int LO_FN(load_prog)(uint32_t wavelet, const lo_user_step* up,
                            size_t nup, LO_FN(lo_step) * prog, size_t* np,
                            size_t* width) {
  lo_prog_row rows[LO_MAX_STEPS];
  size_t k, n;
  int rc = lo_rows(wavelet, up, nup, rows, &n, width);
  if (rc) return rc;
  for (k = 0; k < n; ++k) LO_FN(resolve)(&rows[k], &prog[k]);
  *np = n;
  return 0;
}

int LO_FN(lo_fixed_apply)(uint32_t wavelet, const lo_user_step* up,
                          size_t nup, uint32_t tf, uint32_t bc, T* s, T* d,
                          size_t ns, size_t nd) {
  LO_FN(lo_step) prog[LO_MAX_STEPS];
  size_t np, width;
  int err = 0, rc;
  if (tf > 3 || bc > 4) return 1;
  rc = LO_FN(load_prog)(wavelet, up, nup, prog, &np, &width);
  if (rc) return rc;
  LO_FN(fixed)(prog, np, (int)tf, (int)bc, s, d, ns, nd, &err);
  return err ? 2 : 0;
}

/* Separable nD transform (general_nd, src/lifted-drivers-inl.hpp:417-486):
 * for each axis in the caller's order, the full multi-level 1D transform of
 * every line; the first axis reads `in`, later axes work in place on `out`.
 * A level of 0 means max_level(width, len) (:463). */
int LO_FN(lo_sep)(uint32_t wavelet, const lo_user_step* up, size_t nup,
                  size_t width_in, uint32_t tf, uint32_t bc, size_t ndim,
                  const size_t* shape, const ptrdiff_t* sin,
                  const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                  const size_t* levels, const T* in, T* out) {
  LO_FN(lo_step) prog[LO_MAX_STEPS];
  size_t np, width, iax, total = 1, d;
  int err = 0, rc;
  T *w0, *w1;
  size_t maxlen = 1;
  if (tf > 3 || bc > 4 || ndim == 0 || ndim > 32) return 1;
  rc = LO_FN(load_prog)(wavelet, up, nup, prog, &np, &width);
  if (rc) return rc;
  if (up) width = width_in;
  for (iax = 0; iax < naxes; ++iax)
    if (axes[iax] >= ndim) return 1;
  for (d = 0; d < ndim; ++d) {
    total *= shape[d];
    if (shape[d] > maxlen) maxlen = shape[d];
  }
  if (total == 0) return 0;
  for (iax = 0; iax < naxes; ++iax) {
    size_t lv = levels[iax];
    /* max_level(1, n) never returns in the reference */
    if (lv == 0 && width == 1) return 2;
    if (lv > 62) return 1;
  }
  w0 = (T*)malloc(sizeof(T) * (4 * maxlen + 8));
  w1 = (T*)malloc(sizeof(T) * (4 * maxlen + 8));
  if (!w0 || !w1) { free(w0); free(w1); return 1; }
  for (iax = 0; iax < naxes; ++iax) {
    size_t ax = axes[iax];
    size_t len = shape[ax];
    size_t lv = levels[iax];
    size_t nlines = total / len, li;
    size_t idx[32];
    if (lv == 0) lv = lo_max_level(width, len);
    memset(idx, 0, sizeof(idx));
    for (li = 0; li < nlines; ++li) {
      ptrdiff_t oi = 0, oo = 0;
      for (d = 0; d < ndim; ++d) {
        oi += (ptrdiff_t)idx[d] * sin[d];
        oo += (ptrdiff_t)idx[d] * sout[d];
      }
      if (iax == 0)
        LO_FN(line)(prog, np, (int)tf, (int)bc, in + oi, sin[ax], out + oo,
                    sout[ax], len, lv, w0, w1, &err);
      else
        LO_FN(line)(prog, np, (int)tf, (int)bc, out + oo, sout[ax], out + oo,
                    sout[ax], len, lv, w0, w1, &err);
      /* advance the multi-index over every dim except ax */
      for (d = ndim; d-- > 0;) {
        if (d == ax) continue;
        if (++idx[d] < shape[d]) break;
        idx[d] = 0;
      }
    }
  }
  free(w0);
  free(w1);
  return err ? 2 : 0;
}

/* Non-separable (Mallat) nD transform (general_nd,
 * src/lifted-drivers-inl.hpp:488-610): per level, one single-level pass per
 * axis over the shrinking approximation corner.  Reverse-stepping
 * transforms first copy in -> out and then work in place. */
int LO_FN(lo_nonsep)(uint32_t wavelet, const lo_user_step* up, size_t nup,
                     size_t width_in, uint32_t tf, uint32_t bc, size_t ndim,
                     const size_t* shape, const ptrdiff_t* sin,
                     const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                     size_t level, const T* in, T* out) {
  LO_FN(lo_step) prog[LO_MAX_STEPS];
  size_t np, width, iax, total = 1, d, lvl, ilvl;
  int err = 0, rc;
  T *w0, *w1;
  size_t maxlen = 1;
  size_t shp[64][32];
  const T* src = in;
  const ptrdiff_t* ssrc = sin;
  int fwd_loop = (tf == LO_TF_F || tf == LO_TF_IA);
  if (tf > 3 || bc > 4 || ndim == 0 || ndim > 32 || naxes == 0) return 1;
  rc = LO_FN(load_prog)(wavelet, up, nup, prog, &np, &width);
  if (rc) return rc;
  if (up) width = width_in;
  for (iax = 0; iax < naxes; ++iax)
    if (axes[iax] >= ndim) return 1;
  for (d = 0; d < ndim; ++d) {
    total *= shape[d];
    if (shape[d] > maxlen) maxlen = shape[d];
  }
  if (total == 0) return 0;
  lvl = level;
  if (lvl == 0) {
    size_t min_n;
    if (width == 1) return 2;
    min_n = shape[axes[0]];
    for (iax = 1; iax < naxes; ++iax)
      if (shape[axes[iax]] < min_n) min_n = shape[axes[iax]];
    lvl = lo_max_level(width, min_n);
    if (lvl == 0) return 2; /* the reference indexes an empty level list */
  }
  if (lvl > 62) return 1;
  for (d = 0; d < ndim; ++d) shp[0][d] = shape[d];
  for (ilvl = 1; ilvl < lvl; ++ilvl) {
    for (d = 0; d < ndim; ++d) shp[ilvl][d] = shp[ilvl - 1][d];
    for (iax = 0; iax < naxes; ++iax) {
      size_t a = axes[iax];
      shp[ilvl][a] = shp[ilvl - 1][a] - shp[ilvl - 1][a] / 2;
    }
  }
  w0 = (T*)malloc(sizeof(T) * (4 * maxlen + 8));
  w1 = (T*)malloc(sizeof(T) * (4 * maxlen + 8));
  if (!w0 || !w1) { free(w0); free(w1); return 1; }
  if (!fwd_loop && (const void*)in != (const void*)out) {
    /* copy_inout over the full shape (:542-567) */
    size_t idx[32], li;
    memset(idx, 0, sizeof(idx));
    for (li = 0; li < total; ++li) {
      ptrdiff_t oi = 0, oo = 0;
      for (d = 0; d < ndim; ++d) {
        oi += (ptrdiff_t)idx[d] * sin[d];
        oo += (ptrdiff_t)idx[d] * sout[d];
      }
      out[oo] = in[oi];
      for (d = ndim; d-- > 0;) {
        if (++idx[d] < shape[d]) break;
        idx[d] = 0;
      }
    }
    src = out;
    ssrc = sout;
  }
  for (ilvl = 0; ilvl < lvl; ++ilvl) {
    const size_t* sh = fwd_loop ? shp[ilvl] : shp[lvl - 1 - ilvl];
    size_t sub_total = 1;
    for (d = 0; d < ndim; ++d) sub_total *= sh[d];
    for (iax = 0; iax < naxes; ++iax) {
      size_t ax = axes[iax];
      size_t len = sh[ax];
      size_t nlines = sub_total / len, li;
      size_t idx[32];
      const T* tsrc = (iax == 0) ? src : out;
      const ptrdiff_t* tstr = (iax == 0) ? ssrc : sout;
      /* Lines along an axis whose output stride is 1 always take the Along
       * form here (out_dim_contiguous, :580,595-602). */
      int saved_order = lo_fold_across;
      if (sout[ax] == 1) lo_fold_across = 0;
      memset(idx, 0, sizeof(idx));
      for (li = 0; li < nlines; ++li) {
        ptrdiff_t oi = 0, oo = 0;
        for (d = 0; d < ndim; ++d) {
          oi += (ptrdiff_t)idx[d] * tstr[d];
          oo += (ptrdiff_t)idx[d] * sout[d];
        }
        LO_FN(line)(prog, np, (int)tf, (int)bc, tsrc + oi, tstr[ax], out + oo,
                    sout[ax], len, 1, w0, w1, &err);
        for (d = ndim; d-- > 0;) {
          if (d == ax) continue;
          if (++idx[d] < sh[d]) break;
          idx[d] = 0;
        }
      }
      lo_fold_across = saved_order;
    }
    src = out;
    ssrc = sout;
  }
  free(w0);
  free(w1);
  return err ? 2 : 0;
}

#undef LO_FN
#undef LO_CAT
#undef LO_CAT2
