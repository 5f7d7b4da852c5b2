// Register-blocked lifting kernel of the B200 DWT (the fast path).
//
// Each thread owns a contiguous chunk of P (s, d) pairs of one line in
// registers.  Every lifting step is a register update of the chunk; the few
// neighbour values a step needs from the adjacent chunks cross through a
// double-buffered shared-memory mailbox (one block barrier per step).  The
// split of a level's approximation band into the next level's (s, d) pairs
// is a register renaming, so consecutive levels run without touching memory;
// each level's detail band is stored as soon as it is final.  When a level's
// chunk would fall below the wavelet's reach, the remaining (small) levels
// finish in shared memory with the exact general step code.
//
// The step structure (kind, updated band, offset, tap count, sign) is a
// compile-time function of the catalogue wavelet and transform; the
// coefficients come from the host-resolved program.  Arithmetic per element
// is exactly the reference's Across form (src/lifted-steps-inl.hpp:500-615,
// 754-885, 1011-1126): sequential fused multiply-adds over the taps, repeat
// steps summing their taps first.  This kernel serves the Zero boundary,
// where taps outside the band are skipped and the adjoint folds
// (src/lifted-steps-inl.hpp:529-546, 576-593) never write, so chunk-local
// skipping at the band ends reproduces the reference element for element.
//
// Modes:
//   whole line  a CTA holds whole lines (one level-0 line = TPL chunks)
//   tile        a CTA holds a window [tile start - halo, tile end + halo) of
//               a long line and runs its first levels; only the tile interior
//               is stored, the level's approximation band goes to a scratch
//               band buffer that a whole-line launch finishes.
// Thread mapping:
//   contiguous  thread = line * TPL + chunk (lines along a unit-stride axis)
//   strided     thread = chunk * 32 + line  (32 adjacent lines per CTA: each
//               load/store instruction covers 32 neighbouring lines)
#pragma once

#include <cstdint>

#include "lw_cache.cuh"
#include "lw_edge.cuh"
#include "lw_lanevec.cuh"
#include "lw_line_kernel.cuh"
#include "lw_types.hpp"

namespace lw {

#ifndef LW_K_GEN
#define LW_K_GEN 0
#define LW_K_UNIT 1
#define LW_K_REPEAT 2
#define LW_K_SCALE 3
#define LW_EVENS 0
#define LW_ODDS 1
#define LW_PM_ADD 0
#define LW_PM_SUB 1
#endif

struct CatShape {
  int kind, target, offset, ntaps, pm;
};
struct CatRange {
  int first, count, width;
};

static constexpr CatShape kShapes[] = {
#define LW_CATALOGUE_SHAPES
#include "wavelet_catalogue.inc"
#undef LW_CATALOGUE_SHAPES
};
static constexpr CatRange kRanges[] = {
#define LW_CATALOGUE_RANGES
#include "wavelet_catalogue.inc"
#undef LW_CATALOGUE_RANGES
};

// One step of catalogue wavelet `wi` (catalogue index) for transform `op`,
// in execution order: the compile-time counterpart of resolve_program().
struct CStep {
  int kind, y_is_d, off, ntaps, sub, left, right;
};

constexpr CStep cstep(int wi, int op, int k) {
  const bool normal = (op == TF_F || op == TF_I);
  const bool fwd_tf = (op == TF_F || op == TF_FA);
  const bool fwd_loop = (op == TF_F || op == TF_IA);
  const int cnt = kRanges[wi].count;
  const CatShape s = kShapes[kRanges[wi].first + (fwd_loop ? k : cnt - 1 - k)];
  CStep c{s.kind, 0, 0, s.kind == K_UNIT ? 1 : s.ntaps, 0, 0, 0};
  if (s.kind == K_SCALE) return c;
  const int target = normal ? 1 : 0;
  c.y_is_d = (s.target == target) ? 1 : 0;
  c.off = normal ? s.offset : -(c.ntaps - 1 + s.offset);
  c.sub = (s.kind == K_UNIT) ? (fwd_tf ? s.pm : !s.pm) : (fwd_tf ? 0 : 1);
  c.left = c.off < 0 ? -c.off : 0;
  c.right = (c.off + c.ntaps - 1) > 0 ? (c.off + c.ntaps - 1) : 0;
  return c;
}

constexpr int cat_nsteps(int wi) { return kRanges[wi].count; }

// Largest distance (in pairs) a step of (wi, op) reaches outside a chunk.
constexpr int cat_reach(int wi, int op) {
  int r = 0;
  for (int k = 0; k < kRanges[wi].count; ++k) {
    const CStep c = cstep(wi, op, k);
    if (c.left > r) r = c.left;
    if (c.right > r) r = c.right;
  }
  return r;
}

// The generic instantiation of the register kernels: one kernel for every
// catalogue wavelet, each step dispatched at run time (DevStep::shape) to
// the compiled code of its shape, out of the distinct (kind, target, offset,
// taps, sign) shapes of all catalogue steps for that transform.
constexpr int WI_GEN = 4096;
// A second generic instantiation of the block-level kernels with a wider
// neighbour exchange (float32 strided passes of wavelets of reach 6-9).
constexpr int WI_GENW = 4097;
constexpr bool is_gen(int wi) { return wi == WI_GEN || wi == WI_GENW; }
constexpr int kNumCatalogue = (int)(sizeof(kRanges) / sizeof(kRanges[0]));
constexpr int kMaxGenShapes = 96;

struct GenShapes {
  CStep s[kMaxGenShapes];
  int n;
};

constexpr bool same_shape(const CStep& a, const CStep& b) {
  return a.kind == b.kind && a.y_is_d == b.y_is_d && a.off == b.off && a.ntaps == b.ntaps &&
         a.sub == b.sub;
}

constexpr GenShapes gen_shapes(int op) {
  GenShapes g{};
  g.n = 0;
  for (int wi = 0; wi < kNumCatalogue; ++wi)
    for (int k = 0; k < kRanges[wi].count; ++k) {
      const CStep c = cstep(wi, op, k);
      if (c.kind == K_SCALE) continue;
      bool found = false;
      for (int i = 0; i < g.n && !found; ++i) found = same_shape(g.s[i], c);
      if (!found && g.n < kMaxGenShapes) g.s[g.n++] = c;
    }
  return g;
}

template <int OP>
struct GenTable {
  static constexpr GenShapes v = gen_shapes(OP);
};

// Reach of the level recursion (the generic kernels compile every level
// down to one pair per chunk; the host bounds the levels by the actual
// wavelet's reach) and register levels of an instantiation.
constexpr int kreach(int wi, int op) { return is_gen(wi) ? 1 : cat_reach(wi, op); }
// Neighbour-exchange width of the block-level register kernels: the
// wavelet's reach, or for the generic instantiation a fixed width (wavelets
// of larger reach stay on the general kernel there).
constexpr int kGenHmax = 5;
constexpr int kGenWideHmax = 9;
constexpr int khmax(int wi, int op) {
  return wi == WI_GEN    ? kGenHmax
         : wi == WI_GENW ? kGenWideHmax
                         : (cat_reach(wi, op) > 0 ? cat_reach(wi, op) : 1);
}

// Halo (pairs, per side) that one level of (wi, op) consumes.
constexpr int cat_level_halo(int wi, int op) {
  int l = 0, r = 0;
  for (int k = 0; k < kRanges[wi].count; ++k) {
    const CStep c = cstep(wi, op, k);
    l += c.left;
    r += c.right;
  }
  return l > r ? l : r;
}

template <typename T>
struct RegParams {
  const T* in;
  T* out;
  T* tmp;                 // tile mode: approximation band of the last level
  int64_t tmp_line;       // tmp element (line L, position p) at
  int64_t tmp_pos;        //   tmp[L * tmp_line + p * tmp_pos]
  LineGeom g;
  int32_t levels;         // whole line: all levels of the pass
  int32_t nreg;           // levels run in registers (the finest ones)
  int32_t tpl;            // chunks per window (threads or warps)
  int32_t lpc;            // contiguous mode: lines per CTA
  int64_t tile;           // tile mode: interior length (level-0 elements)
  int64_t halo;           // tile mode: halo per side, a multiple of 2*P0
  int64_t ntiles;         // tile mode: tiles per line
  int32_t vec;            // contiguous unit-stride rows 16-byte aligned
  int32_t coarse_pitch;   // shared coarse buffer: elements per line (A)
  int32_t coarse_pitch_b; // and of its split buffer (B)
  int32_t l2hint;         // L2 priorities of loads and stores (lw_cache.cuh)
  int32_t bc;             // boundary condition: Zero, or Constant / Symmetric /
                          // Reflect with exact band edges (lw_edge.cuh)
  int32_t pad2_;
  DevProgram<T> prog;
};

namespace reg {

template <typename T>
struct Ctx {
  const RegParams<T>* p;
  T* mb;            // mailbox [2 buffers][2 sides][hmax][nth]
  T* cA;            // coarse buffers
  T* cB;
  int nth, tid, tid_l, tid_r, j, r;
  bool has_l, has_r, line_ok;
  int64_t L, bin, bout, n, e0, tile_lo, tile_hi;
  int buf;
  int64_t nsl, ndl; // band lengths of the current level: s (ceil(m / 2)) and
                    // d (floor(m / 2)) of the level's input band of m
  int mb_bufs;      // mailbox buffers: 2 (alternating, one barrier per
                    // step) or 1 (a second barrier after the reads)
  int bc;           // boundary condition of the pass
  uint64_t pol_st;  // L2 policy of the band stores
};

template <typename VT>
__device__ __forceinline__ VT tap(const VT* xl, const bool* vl, const VT* x,
                                  const VT* xr, const bool* vr, int idx, int P,
                                  int HL, bool& ok, int lim) {
  if (idx < 0) {
    ok = vl[HL + idx];
    return xl[HL + idx];
  }
  if (idx >= P) {
    ok = vr[idx - P];
    return xr[idx - P];
  }
  ok = idx < lim;  // lim = P unless the band ends inside this chunk
  return x[idx];
}

// y[0..P) updated from x with one step of compile-time shape CS.  EM: the
// band (nb pairs) may end inside a chunk (lines whose length is not a
// multiple of the chunk); in-chunk taps past the end are skipped.
template <typename T, typename VT, int P, int PA, int HMAX, int KIND, int OFF,
          int NT, int SUB, int HL, int HR, bool YD, bool EM = false, bool EDGE = false>
__device__ __forceinline__ void update(VT (&y)[PA], const VT (&x)[PA],
                                       const DevStep<T>& st, Ctx<T>& c,
                                       int64_t gp0, int64_t nb) {
  static_assert(HL <= P && HR <= P, "step reaches past the neighbour chunk");
  // taps count inside the source band: s (YD: y is d) or d, which differ in
  // length by one on a band of odd length
  int lim = P;
  int64_t nx = nb;
  if constexpr (EM) {
    nx = YD ? c.nsl : c.ndl;
    const int64_t rem = nx - gp0;
    lim = rem >= P ? P : (rem > 0 ? (int)rem : 0);
  }
  // Constant / Symmetric / Reflect: the chunks holding a band end redo
  // that edge around the Zero update (lw_edge.cuh)
  constexpr int E = P < edge::kEdge ? P : edge::kEdge;
  const bool fix = EDGE && !EM && c.bc != BC_ZERO && c.line_ok;
  const bool efront = fix && gp0 == 0;
  const bool eback = fix && gp0 + P == nb;
  VT sf[HL > 0 ? HL : 1], sb[HR > 0 ? HR : 1];
  const DevProgram<T>& prog = c.p->prog;
  const int nth = c.nth;
  VT* mb = reinterpret_cast<VT*>(c.mb);
  VT* mb_first = mb + (int64_t)((c.buf * 2 + 0) * HMAX) * nth;
  VT* mb_last = mb + (int64_t)((c.buf * 2 + 1) * HMAX) * nth;
#pragma unroll
  for (int h = 0; h < HR; ++h) mb_first[h * nth + c.tid] = x[h];
#pragma unroll
  for (int h = 0; h < HL; ++h) mb_last[h * nth + c.tid] = x[P - HL + h];
  __syncthreads();
  if (c.mb_bufs == 2) c.buf ^= 1;
  if constexpr (EDGE) {
    if (efront) edge::call<P, E, false>(st, prog, c.bc, false, y, x, sf, gp0, nb, HL, HR);
    if (eback) edge::call<P, E, true>(st, prog, c.bc, false, y, x, sb, gp0, nb, HL, HR);
  }
  VT xl[HL > 0 ? HL : 1], xr[HR > 0 ? HR : 1];
  bool vl[HL > 0 ? HL : 1], vr[HR > 0 ? HR : 1];
#pragma unroll
  for (int h = 0; h < HL; ++h) {
    xl[h] = c.has_l ? mb_last[h * nth + c.tid_l] : vzero<VT>();
    vl[h] = (gp0 - HL + h) >= 0;
  }
#pragma unroll
  for (int h = 0; h < HR; ++h) {
    xr[h] = c.has_r ? mb_first[h * nth + c.tid_r] : vzero<VT>();
    vr[h] = (gp0 + P + h) < nx;
  }
  if (c.mb_bufs == 1) __syncthreads();  // the mailbox is read before the next step writes it
#pragma unroll
  for (int i = 0; i < P; ++i) {
    VT yi = y[i];
    if constexpr (KIND == K_GEN) {
#pragma unroll
      for (int k = 0; k < NT; ++k) {
        bool ok;
        const VT v = tap(xl, vl, x, xr, vr, i + OFF + k, P, HL, ok, lim);
        const VT f = vfop(SUB, st.c[k], v, yi);
        yi = ok ? f : yi;
      }
    } else if constexpr (KIND == K_REPEAT) {
      bool ok;
      VT v = tap(xl, vl, x, xr, vr, i + OFF, P, HL, ok, lim);
      VT x0 = ok ? v : vzero<VT>();
#pragma unroll
      for (int k = 1; k < NT; ++k) {
        v = tap(xl, vl, x, xr, vr, i + OFF + k, P, HL, ok, lim);
        x0 = ok ? vadd(x0, v) : x0;
      }
      yi = vfop(SUB, st.c[0], x0, yi);
    } else {  // unit
      bool ok;
      const VT v = tap(xl, vl, x, xr, vr, i + OFF, P, HL, ok, lim);
      const VT f = SUB ? vsub(yi, v) : vadd(yi, v);
      yi = ok ? f : yi;
    }
    y[i] = yi;
  }
  if constexpr (EDGE) {
    if (efront) edge::call<P, E, false>(st, prog, c.bc, true, y, x, sf, gp0, nb, HL, HR);
    if (eback) edge::call<P, E, true>(st, prog, c.bc, true, y, x, sb, gp0, nb, HL, HR);
  }
}

// Generic instantiation: one step's update dispatched on its shape index
// (shapes wider than P pairs or than the exchange width are not compiled;
// the host never runs them).  Every thread takes the same branch.
template <typename T, typename VT, int OP, int P, int PA, int HMAX, int I, bool EM = false>
__device__ __forceinline__ void gen_update(int shape, VT (&s)[PA], VT (&d)[PA],
                                           const DevStep<T>& st, Ctx<T>& c, int64_t gp0,
                                           int64_t nb) {
  if constexpr (I < GenTable<OP>::v.n) {
    if (shape == I) {
      constexpr CStep cs = GenTable<OP>::v.s[I];
      if constexpr (cs.left <= P && cs.right <= P && cs.left <= HMAX && cs.right <= HMAX) {
        if constexpr (cs.y_is_d)
          update<T, VT, P, PA, HMAX, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, true,
                 EM>(d, s, st, c, gp0, nb);
        else
          update<T, VT, P, PA, HMAX, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, false,
                 EM>(s, d, st, c, gp0, nb);
      }
      return;
    }
    gen_update<T, VT, OP, P, PA, HMAX, I + 1, EM>(shape, s, d, st, c, gp0, nb);
  }
}

template <typename T, typename VT, int WI, int OP, int K, int P, int PA,
          int HMAX, bool EM = false, bool EDGE = false>
__device__ __forceinline__ void steps(VT (&s)[PA], VT (&d)[PA], Ctx<T>& c,
                                      int64_t gp0, int64_t nb) {
  if constexpr (is_gen(WI)) {
    if constexpr (K == 0) {
      const DevProgram<T>& prog = c.p->prog;
      for (int k = 0; k < prog.nsteps; ++k) {
        const DevStep<T>& st = prog.st[k];
        if (st.kind == K_SCALE) {
          const T sm = st.sm, dm = st.dm;
#pragma unroll
          for (int i = 0; i < P; ++i) {
            s[i] = vmul(s[i], sm);
            d[i] = vmul(d[i], dm);
          }
        } else {
          gen_update<T, VT, OP, P, PA, HMAX, 0, EM>(st.shape, s, d, st, c, gp0, nb);
        }
      }
    }
  } else if constexpr (K < cat_nsteps(WI)) {
    constexpr CStep cs = cstep(WI, OP, K);
    const DevStep<T>& st = c.p->prog.st[K];
    if constexpr (cs.kind == K_SCALE) {
      const T sm = st.sm, dm = st.dm;
#pragma unroll
      for (int i = 0; i < P; ++i) {
        s[i] = vmul(s[i], sm);
        d[i] = vmul(d[i], dm);
      }
    } else if constexpr (cs.y_is_d) {
      update<T, VT, P, PA, HMAX, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left,
             cs.right, true, EM, EDGE>(d, s, st, c, gp0, nb);
    } else {
      update<T, VT, P, PA, HMAX, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left,
             cs.right, false, EM, EDGE>(s, d, st, c, gp0, nb);
    }
    steps<T, VT, WI, OP, K + 1, P, PA, HMAX, EM, EDGE>(s, d, c, gp0, nb);
  }
}

// The steps of one level in an exact-edge instantiation: a warp with a
// lane on a band end runs the edge-aware step code, every other warp the
// Zero step code, which has no call to the edge routine and compiles like
// the Zero kernels' (the call otherwise constrains the code around it).
// The choice is warp-uniform, and both forms take the same barriers.
template <typename T, typename VT, int WI, int OP, int P, int PA, int HMAX, bool EM, bool EDGE>
__device__ __forceinline__ void steps_sel(VT (&s)[PA], VT (&d)[PA], Ctx<T>& c, int64_t gp0,
                                          int64_t nb) {
  if constexpr (EDGE) {
    const bool mine = c.bc != BC_ZERO && c.line_ok && (gp0 == 0 || gp0 + P == nb);
    if (__any_sync(0xffffffffu, mine))
      steps<T, VT, WI, OP, 0, P, PA, HMAX, EM, true>(s, d, c, gp0, nb);
    else
      steps<T, VT, WI, OP, 0, P, PA, HMAX, EM, false>(s, d, c, gp0, nb);
  } else {
    steps<T, VT, WI, OP, 0, P, PA, HMAX, EM, false>(s, d, c, gp0, nb);
  }
}

// Stores P consecutive band values v[0..P) at line positions pos0.. of the
// destination (vectorised for unit-stride aligned rows; with V lines per
// lane, one V-wide store per position covers the lane's adjacent lines).
template <typename T, typename VT, int P, int PA>
__device__ __forceinline__ void store_run(const VT (&v)[PA], Ctx<T>& c,
                                          int64_t pos0) {
  const RegParams<T>& p = *c.p;
  T* o = p.out + c.bout + pos0 * p.g.sout;
  if constexpr (sizeof(VT) == sizeof(T)) {
    constexpr int VW = 16 / (int)sizeof(T);
    if constexpr (P % VW == 0) {
      if (p.vec && ((pos0 % VW) == 0)) {
#pragma unroll
        for (int i = 0; i < P; i += VW) {
          if constexpr (sizeof(T) == 4) {
            st_hint(o + i, make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]), c.pol_st);
          } else {
            st_hint(o + i, make_double2(v[i], v[i + 1]), c.pol_st);
          }
        }
        return;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < P; ++i) st_hint(o + i * p.g.sout, v[i], c.pol_st);
}

// store_run limited to the first `lim` positions (a band ending inside the
// chunk), one store per position.
template <typename T, typename VT, int P, int PA>
__device__ __forceinline__ void store_first(const VT (&v)[PA], Ctx<T>& c, int64_t pos0, int lim) {
  const RegParams<T>& p = *c.p;
  T* o = p.out + c.bout + pos0 * p.g.sout;
#pragma unroll
  for (int i = 0; i < P; ++i)
    if (i < lim) st_hint(o + i * p.g.sout, v[i], c.pol_st);
}

template <typename T>
__device__ __forceinline__ bool chunk_stored(const Ctx<T>& c) {
  return c.line_ok && c.e0 >= c.tile_lo && c.e0 < c.tile_hi;
}

// Band lengths of level lv of a line of n samples: its input band has
// ceil(n / 2^lv) samples, split into ceil and floor halves.
template <typename T>
__device__ __forceinline__ void level_lengths(Ctx<T>& c, int lv) {
  const int64_t m = (c.n + ((int64_t)1 << lv) - 1) >> lv;
  c.ndl = m >> 1;
  c.nsl = m - c.ndl;
}

__device__ __forceinline__ int chunk_lim(int64_t len, int64_t gp0, int P) {
  const int64_t rem = len - gp0;
  return rem >= P ? P : (rem > 0 ? (int)rem : 0);
}

// Forward-stepping register levels (Forward, InverseAdjoint).
// EM: lines whose length is not a multiple of the chunk: a band ends inside
// a chunk, whose stores stop there; at a level whose input band is odd the
// s band is one longer than the d band.
template <typename T, typename VT, int V, int WI, int OP, int P0, int HMAX,
          int LV, bool TILE, bool EM = false, bool EDGE = false>
__device__ __forceinline__ void fwd_levels(VT (&s)[P0], VT (&d)[P0],
                                           Ctx<T>& c) {
  constexpr int P = P0 >> LV;
  if constexpr (P >= 1 && P >= kreach(WI, OP) && LV < MAX_LEVELS) {
    if (LV < c.p->nreg) {
      const int64_t nb = c.n >> (LV + 1);
      const int64_t gp0 = c.e0 >> (LV + 1);
      int lim = P;  // s values of this chunk inside the band
      if constexpr (EM) {
        level_lengths(c, LV);
        lim = chunk_lim(c.nsl, gp0, P);
      }
      steps_sel<T, VT, WI, OP, P, P0, HMAX, EM, EDGE>(s, d, c, gp0, nb);
      if (chunk_stored(c)) {
        if constexpr (EM) store_first<T, VT, P, P0>(d, c, c.nsl + gp0, chunk_lim(c.ndl, gp0, P));
        else store_run<T, VT, P, P0>(d, c, nb + gp0);
      }
      if (LV + 1 == c.p->nreg) {
        // hand the approximation band on
        if (TILE && c.p->nreg < c.p->levels) {
          if (chunk_stored(c)) {
            T* t = c.p->tmp + c.L * c.p->tmp_line;
#pragma unroll
            for (int i = 0; i < P; ++i)
              if (!EM || i < lim) st_hint(t + (gp0 + i) * c.p->tmp_pos, s[i], c.pol_st);
          }
        } else if (TILE) {
          if (chunk_stored(c)) {
            if constexpr (EM) store_first<T, VT, P, P0>(s, c, gp0, lim);
            else store_run<T, VT, P, P0>(s, c, gp0);
          }
        } else if (c.p->nreg == c.p->levels) {
          if (c.line_ok) {
            if constexpr (EM) store_first<T, VT, P, P0>(s, c, gp0, lim);
            else store_run<T, VT, P, P0>(s, c, gp0);
          }
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            T* a = c.cA + (int64_t)(c.j * V + v) * c.p->coarse_pitch;
#pragma unroll
            for (int i = 0; i < P; ++i) a[gp0 + i] = vlane(s[i], v);
          }
        }
        return;
      }
#pragma unroll
      for (int i = 0; i < P / 2; ++i) {
        d[i] = s[2 * i + 1];
        s[i] = s[2 * i];
      }
      fwd_levels<T, VT, V, WI, OP, P0, HMAX, LV + 1, TILE, EM, EDGE>(s, d, c);
    }
  }
}

// Reverse-stepping register levels (Inverse, ForwardAdjoint), coarsest
// register level first.
template <typename T, typename VT, int V, int WI, int OP, int P0, int HMAX,
          int LV, bool TILE, bool EDGE = false>
__device__ __forceinline__ void rev_levels(VT (&s)[P0], VT (&d)[P0],
                                           Ctx<T>& c) {
  constexpr int P = P0 >> LV;
  if constexpr (LV >= 0) {
    if constexpr (P >= 1 && P >= kreach(WI, OP)) {
      if (LV < c.p->nreg) {
        const RegParams<T>& p = *c.p;
        const int64_t nb = c.n >> (LV + 1);
        const int64_t gp0 = c.e0 >> (LV + 1);
        if (LV + 1 == p.nreg) {  // approximation band of the coarsest level
          if (TILE && p.nreg < p.levels) {
            const T* t = p.tmp + c.L * p.tmp_line;
#pragma unroll
            for (int i = 0; i < P; ++i) {
              const int64_t q = gp0 + i;
              s[i] = (c.line_ok && q >= 0 && q < nb)
                         ? *reinterpret_cast<const VT*>(t + q * p.tmp_pos)
                         : vzero<VT>();
            }
          } else if (p.nreg == p.levels) {
#pragma unroll
            for (int i = 0; i < P; ++i) {
              const int64_t q = gp0 + i;
              s[i] = (c.line_ok && q >= 0 && q < nb)
                         ? *reinterpret_cast<const VT*>(p.in + c.bin + q * p.g.sin)
                         : vzero<VT>();
            }
          } else {
#pragma unroll
            for (int i = 0; i < P; ++i) {
              if constexpr (V == 1) {
                s[i] = c.cA[(int64_t)c.j * p.coarse_pitch + gp0 + i];
              } else {
                const T* a0 = c.cA + (int64_t)(c.j * V) * p.coarse_pitch;
                s[i] = VT{a0[gp0 + i], a0[p.coarse_pitch + gp0 + i]};
              }
            }
          }
        }
#pragma unroll
        for (int i = 0; i < P; ++i) {
          const int64_t q = gp0 + i;
          d[i] = (c.line_ok && q >= 0 && q < nb)
                     ? *reinterpret_cast<const VT*>(p.in + c.bin + (nb + q) * p.g.sin)
                     : vzero<VT>();
        }
        steps_sel<T, VT, WI, OP, P, P0, HMAX, false, EDGE>(s, d, c, gp0, nb);
        if constexpr (LV == 0) {
          if (chunk_stored(c)) {
            T* o = p.out + c.bout + c.e0 * p.g.sout;
            constexpr int VW = 16 / (int)sizeof(T);
            if (V == 1 && p.vec && (c.e0 % VW) == 0) {
#pragma unroll
              for (int i = 0; i < P; i += VW / 2) {
                if constexpr (sizeof(T) == 4) {
                  st_hint(o + 2 * i,
                          make_float4(vlane(s[i], 0), vlane(d[i], 0), vlane(s[i + 1], 0),
                                      vlane(d[i + 1], 0)),
                          c.pol_st);
                } else {
                  st_hint(o + 2 * i, make_double2(vlane(s[i], 0), vlane(d[i], 0)), c.pol_st);
                }
              }
            } else {
#pragma unroll
              for (int i = 0; i < P; ++i) {
                st_hint(o + (2 * i) * p.g.sout, s[i], c.pol_st);
                st_hint(o + (2 * i + 1) * p.g.sout, d[i], c.pol_st);
              }
            }
          }
        } else {
#pragma unroll
          for (int i = P - 1; i >= 0; --i) {
            s[2 * i + 1] = d[i];
            s[2 * i] = s[i];
          }
        }
      }
      if constexpr (LV > 0)
        rev_levels<T, VT, V, WI, OP, P0, HMAX, LV - 1, TILE, EDGE>(s, d, c);
    } else if constexpr (LV > 0) {
      rev_levels<T, VT, V, WI, OP, P0, HMAX, LV - 1, TILE, EDGE>(s, d, c);
    }
  }
}

}  // namespace reg

// Number of levels the register path can run with P0 pairs per chunk.
constexpr int reg_max_levels(int wi, int op, int p0) {
  int lv = 0;
  const int reach = kreach(wi, op);
  for (int p = p0; p >= 1 && p >= reach && lv < MAX_LEVELS; p >>= 1) ++lv;
  return lv;
}

// V: adjacent lines per lane (strided mode only; 2 packs float pairs into
// FP32x2 arithmetic and 8-byte accesses).  lines per CTA = lpc * V.
// EDGE: the instantiation for the Constant, Symmetric and Reflect
// boundaries (exact band edges, lw_edge.cuh); Zero passes run the one
// without that code.
template <typename T, int WI, int OP, int P0, bool STRIDED, bool TILE, int V, bool EDGE = false>
__global__ void __launch_bounds__(512)
    reg_kernel(const __grid_constant__ RegParams<T> p) {
  using VT = typename LaneVec<T, V>::type;
  static_assert(V == 1 || STRIDED, "vector lanes need the strided mapping");
  constexpr int HMAX = khmax(WI, OP);
  constexpr bool FWD = (OP == TF_F || OP == TF_IA);
  extern __shared__ __align__(16) unsigned char lw_reg_smem[];
  pdl_wait();  // the previous kernel's results (no global access before)
  pdl_trigger();
  reg::Ctx<T> c;
  c.p = &p;
  c.nth = blockDim.x;
  c.tid = threadIdx.x;
  c.mb = reinterpret_cast<T*>(lw_reg_smem);
  // mailbox: 4 * HMAX * nth lane values, then the coarse buffers
  c.cA = reinterpret_cast<T*>(reinterpret_cast<VT*>(c.mb) + 4 * HMAX * c.nth);
  c.cA = reinterpret_cast<T*>(
      (reinterpret_cast<uintptr_t>(c.cA) + 15) & ~uintptr_t(15));
  const int lpc = p.lpc;               // lanes (line groups) per CTA row
  const int lines_cta = lpc * V;
  c.cB = c.cA + (int64_t)lines_cta * p.coarse_pitch;
  if (STRIDED) {
    c.j = c.tid % lpc;
    c.r = c.tid / lpc;
    c.tid_l = c.tid - lpc;
    c.tid_r = c.tid + lpc;
  } else {
    c.j = c.tid / p.tpl;
    c.r = c.tid - c.j * p.tpl;
    c.tid_l = c.tid - 1;
    c.tid_r = c.tid + 1;
  }
  c.has_l = c.r > 0;
  c.has_r = c.r < p.tpl - 1;
  c.buf = 0;
  c.mb_bufs = 2;
  c.bc = p.bc;
  c.pol_st = l2_store_policy(p.l2hint);
  int64_t tile_idx = 0, group = blockIdx.x;
  if (TILE) {
    tile_idx = blockIdx.x % p.ntiles;
    group = blockIdx.x / p.ntiles;
  }
  c.L = group * lines_cta + (int64_t)c.j * V;
  c.line_ok = c.L < p.g.nlines;  // V lines together (nlines % V == 0)
  c.bin = 0;
  c.bout = 0;
  if (c.line_ok) line_base(p.g, c.L, c.bin, c.bout);
  c.n = p.g.n;
  const int64_t wstart = TILE ? tile_idx * p.tile - p.halo : 0;
  c.e0 = wstart + (int64_t)2 * P0 * c.r;
  if (TILE) {
    c.tile_lo = tile_idx * p.tile;
    c.tile_hi = c.tile_lo + p.tile < c.n ? c.tile_lo + p.tile : c.n;
  } else {
    c.tile_lo = 0;
    c.tile_hi = c.n;
  }

  VT s[P0], d[P0];
  if constexpr (FWD) {
    const bool in_band = c.line_ok && c.e0 >= 0 && c.e0 < c.n;
    const T* src = p.in + c.bin + c.e0 * p.g.sin;
    constexpr int VW = 16 / (int)sizeof(T);
    if (V == 1 && in_band && p.vec && (c.e0 % VW) == 0) {
#pragma unroll
      for (int e = 0; e < 2 * P0; e += VW) {
        if constexpr (V == 1 && sizeof(T) == 4) {
          const float4 v = *reinterpret_cast<const float4*>(src + e);
          s[e / 2] = v.x;
          d[e / 2] = v.y;
          s[e / 2 + 1] = v.z;
          d[e / 2 + 1] = v.w;
        } else if constexpr (V == 1) {
          const double2 v = *reinterpret_cast<const double2*>(src + e);
          s[e / 2] = v.x;
          d[e / 2] = v.y;
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < P0; ++i) {
        s[i] = in_band ? *reinterpret_cast<const VT*>(src + (2 * i) * p.g.sin)
                       : vzero<VT>();
        d[i] = in_band ? *reinterpret_cast<const VT*>(src + (2 * i + 1) * p.g.sin)
                       : vzero<VT>();
      }
    }
    reg::fwd_levels<T, VT, V, WI, OP, P0, HMAX, 0, TILE, false, EDGE>(s, d, c);
    if constexpr (!TILE) {
      if (p.nreg < p.levels) {
        __syncthreads();
        const int64_t m = c.n >> p.nreg;
        coarse_forward(p.prog, p.bc, c.cA, p.coarse_pitch, c.cB,
                       p.coarse_pitch_b, lines_cta, m, p.levels - p.nreg);
        // store the coarse region [0, m) of every line of the CTA
        const int64_t tot = (int64_t)lines_cta * m;
        for (int64_t f = c.tid; f < tot; f += c.nth) {
          int jj;
          int64_t i;
          if (STRIDED) {
            i = f / lines_cta;
            jj = (int)(f - i * lines_cta);
          } else {
            jj = (int)(f / m);
            i = f - (int64_t)jj * m;
          }
          const int64_t LL = group * lines_cta + jj;
          if (LL < p.g.nlines) {
            int64_t bi, bo;
            line_base(p.g, LL, bi, bo);
            p.out[bo + i * p.g.sout] = c.cA[(int64_t)jj * p.coarse_pitch + i];
          }
        }
      }
    }
  } else {
    if constexpr (!TILE) {
      if (p.nreg < p.levels) {
        const int64_t m = c.n >> p.nreg;
        const int64_t tot = (int64_t)lines_cta * m;
        for (int64_t f = c.tid; f < tot; f += c.nth) {
          int jj;
          int64_t i;
          if (STRIDED) {
            i = f / lines_cta;
            jj = (int)(f - i * lines_cta);
          } else {
            jj = (int)(f / m);
            i = f - (int64_t)jj * m;
          }
          const int64_t LL = group * lines_cta + jj;
          T v = T(0);
          if (LL < p.g.nlines) {
            int64_t bi, bo;
            line_base(p.g, LL, bi, bo);
            v = p.in[bi + i * p.g.sin];
          }
          c.cA[(int64_t)jj * p.coarse_pitch + i] = v;
        }
        __syncthreads();
        coarse_reverse(p.prog, p.bc, c.cA, p.coarse_pitch, c.cB,
                       p.coarse_pitch_b, lines_cta, m, p.levels - p.nreg);
      }
    }
    constexpr int TOP = reg_max_levels(WI, OP, P0) - 1;
    reg::rev_levels<T, VT, V, WI, OP, P0, HMAX, TOP, TILE, EDGE>(s, d, c);
  }
}

}  // namespace lw
