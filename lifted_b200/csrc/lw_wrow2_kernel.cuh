// Two-warp-per-row lifting kernel for contiguous float32 rows of 128 * P0
// elements (the warp-per-row kernel, lw_wrow_kernel.cuh, with each row split
// between a pair of warps), persistent, with the next row's copy in flight
// while the current row is lifted.
//
// Half the registers per thread (P0 pairs per lane instead of 2 * P0) let
// an SM hold about twice as many warps, which is what hides the latency of
// the load, shuffle and store phases; the price is one exchange per lifting
// step across the seam between the two warps of a row: lane 31 of the first
// warp and lane 0 of the second swap their edge values through a small
// double-buffered shared-memory mailbox and a 64-thread named barrier.  All
// other neighbour values move by warp shuffles, as in the warp-per-row
// kernel.  Row buffers, the XOR swizzle and the banded output layout are
// those of that kernel with 64 "lanes" (global lane g = 32 * half + lane).
#pragma once

#include <cstdint>

#include "lw_cache.cuh"
#include "lw_wrow_kernel.cuh"

namespace lw {
namespace wrow2 {

constexpr int GL = 64;  // lanes per row

// Swizzle shift of 16-byte unit U of a row written as banded runs with 64
// lanes: the approximation [0, nbl) as runs of nbl/64 elements, each detail
// band [2^k, 2^(k+1)) as runs of 2^k/64.
__device__ __forceinline__ int banded_shift(int U, int nbl) {
  const int e = U * 4;
  const int region = e < nbl ? nbl : (1 << (31 - __clz(e)));
  const int bytes = (region / GL) * 4;
  return bytes >= 1024 ? 3 : bytes >= 512 ? 2 : bytes >= 256 ? 1 : 0;
}

struct Seam {
  float* mb;    // [2 buffers][2 sides][HMAX] of this row
  int half;     // 0: first warp of the row, 1: second
  int lane;
  int bar_id;   // named barrier of the row's 64 threads
  int buf;
};

__device__ __forceinline__ void row_sync(int id) {
  asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
}

// One step over the lane's P pairs: halos by shuffle inside each warp, and
// across the seam of the row's two warps through the mailbox.
// EDGE: the lanes holding the row band's ends (global lanes 0 and 63) redo
// their edge around the Zero update for the Constant, Symmetric and Reflect
// boundaries (lw_edge.cuh).
template <int P, int PA, int HMAX, int KIND, int OFF, int NT, int SUB, int HL, int HR,
          bool EDGE = false>
__device__ __forceinline__ void update(float (&y)[PA], const float (&x)[PA], const DevStep<float>& st,
                                       Seam& sm, const wrow::WEdge<float>* ed = nullptr) {
  static_assert(HL <= P && HR <= P, "step reaches past the neighbour lane");
  float xl[HL > 0 ? HL : 1], xr[HR > 0 ? HR : 1];
#pragma unroll
  for (int h = 0; h < HL; ++h) xl[h] = __shfl_up_sync(wrow::FULL, x[P - HL + h], 1);
#pragma unroll
  for (int h = 0; h < HR; ++h) xr[h] = __shfl_down_sync(wrow::FULL, x[h], 1);
  if (HL > 0 || HR > 0) {
    float* box = sm.mb + sm.buf * 2 * HMAX;
    // side 0: last HL values of the first warp's lane 31; side 1: first HR
    // values of the second warp's lane 0
    if (sm.half == 0 && sm.lane == 31) {
#pragma unroll
      for (int h = 0; h < HL; ++h) box[h] = x[P - HL + h];
    }
    if (sm.half == 1 && sm.lane == 0) {
#pragma unroll
      for (int h = 0; h < HR; ++h) box[HMAX + h] = x[h];
    }
    row_sync(sm.bar_id);
    if (sm.half == 1 && sm.lane == 0) {
#pragma unroll
      for (int h = 0; h < HL; ++h) xl[h] = box[h];
    }
    if (sm.half == 0 && sm.lane == 31) {
#pragma unroll
      for (int h = 0; h < HR; ++h) xr[h] = box[HMAX + h];
    }
    sm.buf ^= 1;
  }
  const int g = sm.half * 32 + sm.lane;
  const bool okl = g > 0, okr = g < GL - 1;
  constexpr int E = P < edge::kEdge ? P : edge::kEdge;
  float sf[HL > 0 ? HL : 1], sb[HR > 0 ? HR : 1];
  bool efront = false, eback = false;
  if constexpr (EDGE) {
    efront = ed->bc != BC_ZERO && !okl;
    eback = ed->bc != BC_ZERO && !okr;
    if (efront)
      edge::call<P, E, false>(st, *ed->prog, ed->bc, false, y, x, sf, 0, ed->nb, HL, HR);
    if (eback)
      edge::call<P, E, true>(st, *ed->prog, ed->bc, false, y, x, sb, ed->nb - P, ed->nb, HL, HR);
  }
#pragma unroll
  for (int i = 0; i < P; ++i) {
    float yi = y[i];
    if constexpr (KIND == K_GEN) {
#pragma unroll
      for (int k = 0; k < NT; ++k) {
        const int idx = i + OFF + k;
        const float v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
        const bool ok = idx < 0 ? okl : (idx >= P ? okr : true);
        const float f = fop(SUB, st.c[k], v, yi);
        yi = ok ? f : yi;
      }
    } else if constexpr (KIND == K_REPEAT) {
      int idx = i + OFF;
      float v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
      bool ok = idx < 0 ? okl : (idx >= P ? okr : true);
      float x0 = ok ? v : 0.0f;
#pragma unroll
      for (int k = 1; k < NT; ++k) {
        idx = i + OFF + k;
        v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
        ok = idx < 0 ? okl : (idx >= P ? okr : true);
        x0 = ok ? x0 + v : x0;
      }
      yi = fop(SUB, st.c[0], x0, yi);
    } else {
      const int idx = i + OFF;
      const float v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
      const bool ok = idx < 0 ? okl : (idx >= P ? okr : true);
      const float f = SUB ? yi - v : yi + v;
      yi = ok ? f : yi;
    }
    y[i] = yi;
  }
  if constexpr (EDGE) {
    if (efront)
      edge::call<P, E, false>(st, *ed->prog, ed->bc, true, y, x, sf, 0, ed->nb, HL, HR);
    if (eback)
      edge::call<P, E, true>(st, *ed->prog, ed->bc, true, y, x, sb, ed->nb - P, ed->nb, HL, HR);
  }
}

template <int WI, int OP, int K, int P, int PA, int HMAX, bool EDGE = false>
__device__ __forceinline__ void steps(float (&s)[PA], float (&d)[PA], const DevProgram<float>& prog,
                                      Seam& sm, const wrow::WEdge<float>* ed = nullptr) {
  if constexpr (K < cat_nsteps(WI)) {
    constexpr CStep cs = cstep(WI, OP, K);
    const DevStep<float>& st = prog.st[K];
    if constexpr (cs.kind == K_SCALE) {
      const float smul = st.sm, dmul = st.dm;
#pragma unroll
      for (int i = 0; i < P; ++i) {
        s[i] = s[i] * smul;
        d[i] = d[i] * dmul;
      }
    } else if constexpr (cs.y_is_d) {
      update<P, PA, HMAX, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, EDGE>(d, s, st, sm,
                                                                                    ed);
    } else {
      update<P, PA, HMAX, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, EDGE>(s, d, st, sm,
                                                                                    ed);
    }
    steps<WI, OP, K + 1, P, PA, HMAX, EDGE>(s, d, prog, sm, ed);
  }
}

template <int WI, int OP, int P0, int HMAX, int LV, bool EDGE = false>
__device__ __forceinline__ void fwd(float (&s)[P0], float (&d)[P0], float* buf,
                                    const DevProgram<float>& prog, int levels, Seam& sm,
                                    int bc = BC_ZERO) {
  constexpr int P = P0 >> LV;
  if constexpr (P >= 1 && P >= cat_reach(WI, OP)) {
    if (LV < levels) {
      constexpr int NB = GL * P;
      const int g = sm.half * 32 + sm.lane;
      const wrow::WEdge<float> ed{&prog, bc, NB};
      steps<WI, OP, 0, P, P0, HMAX, EDGE>(s, d, prog, sm, &ed);
      wrow::write_run<float, P, P>(buf, NB + P * g, d);
      if (LV + 1 == levels) {
        wrow::write_run<float, P, P>(buf, P * g, s);
        return;
      }
#pragma unroll
      for (int i = 0; i < P / 2; ++i) {
        d[i] = s[2 * i + 1];
        s[i] = s[2 * i];
      }
      fwd<WI, OP, P0, HMAX, LV + 1, EDGE>(s, d, buf, prog, levels, sm, bc);
    }
  }
}

template <int WI, int OP, int P0, int HMAX, int LV, bool EDGE = false>
__device__ __forceinline__ void rev(float (&s)[P0], float (&d)[P0], float* buf,
                                    const DevProgram<float>& prog, int levels, Seam& sm,
                                    int bc = BC_ZERO) {
  constexpr int P = P0 >> LV;
  if constexpr (LV >= 0) {
    if constexpr (P >= 1 && P >= cat_reach(WI, OP)) {
      if (LV < levels) {
        constexpr int NB = GL * P;
        const int g = sm.half * 32 + sm.lane;
        if (LV + 1 == levels) wrow::read_run<float, P, P>(buf, P * g, s);
        wrow::read_run<float, P, P>(buf, NB + P * g, d);
        const wrow::WEdge<float> ed{&prog, bc, NB};
        steps<WI, OP, 0, P, P0, HMAX, EDGE>(s, d, prog, sm, &ed);
        if constexpr (LV > 0) {
#pragma unroll
          for (int i = P - 1; i >= 0; --i) {
            s[2 * i + 1] = d[i];
            s[2 * i] = s[i];
          }
        }
      }
    }
    if constexpr (LV > 0) rev<WI, OP, P0, HMAX, LV - 1, EDGE>(s, d, buf, prog, levels, sm, bc);
  }
}

}  // namespace wrow2

// 128 threads = two row slots of 128 * P0 float32 elements, two warps each.
// Persistent: each slot walks rows blockIdx.x*2 + slot, + 2*gridDim.x, ...
// with two row buffers, the next row's cp.async copy in flight while the
// current row is lifted and stored.
// EDGE: the instantiation for the Constant, Symmetric and Reflect
// boundaries (exact band edges; every level's lanes hold the edge reach).
template <int WI, int OP, int P0, bool EDGE = false>
__global__ void __launch_bounds__(128)
    wrow2_kernel(const __grid_constant__ WRowParams<float> p) {
  constexpr int N = 128 * P0;     // row length
  constexpr int UNITS = N / 4;    // 16-byte units per row
  constexpr int HMAX = cat_reach(WI, OP) > 0 ? cat_reach(WI, OP) : 1;
  constexpr bool FWD = (OP == TF_F || OP == TF_IA);
  extern __shared__ __align__(16) unsigned char lw_wrow2_smem[];
  __shared__ float mbox[2][2 * 2 * HMAX];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int rsel = warp >> 1;            // row slot of the CTA
  const int half = warp & 1;
  const int t64 = threadIdx.x & 63;      // thread within the slot
  float* bufs = reinterpret_cast<float*>(lw_wrow2_smem) + (int64_t)rsel * 2 * N;
  wrow2::Seam sm{mbox[rsel], half, lane, 1 + rsel, 0};
  const int nbl = N >> p.levels;
  constexpr int SHA = wrow::swz_shift_bytes(2 * P0 * 4);
  const int g = half * 32 + lane;
  const int64_t step = (int64_t)gridDim.x * 2;
  const uint64_t pol_ld = l2_load_policy(p.l2hint);
  const uint64_t pol_st = l2_store_policy(p.l2hint);

  auto load = [&](int64_t row, float* buf) {
    int64_t bin, bout;
    line_base(p.g, row, bin, bout);
    const float* src = p.in + bin;
#pragma unroll 4
    for (int u = t64; u < UNITS; u += 64) {
      const int sh = FWD ? SHA : wrow2::banded_shift(u, nbl);
      const unsigned saddr = (unsigned)__cvta_generic_to_shared(buf + wrow::swz(u, sh) * 4);
      cp_async16_hint(saddr, src + (int64_t)u * 4, pol_ld);
    }
  };

  int cur = 0;
  int64_t row = (int64_t)blockIdx.x * 2 + rsel;
  pdl_wait();  // the previous kernel's results (no global access before)
  if (row < p.g.nlines) load(row, bufs);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  for (; row < p.g.nlines; row += step) {
    float* buf = bufs + cur * N;
    const int64_t next = row + step;
    if (next >= p.g.nlines) pdl_trigger();  // the slot's last row
    if (next < p.g.nlines) load(next, bufs + (cur ^ 1) * N);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this row's copy
    wrow2::row_sync(sm.bar_id);

    float s[P0], d[P0];
    if constexpr (FWD) {
      float x[2 * P0];
      wrow::read_run<float, 2 * P0, 2 * P0>(buf, 2 * P0 * g, x);
#pragma unroll
      for (int i = 0; i < P0; ++i) {
        s[i] = x[2 * i];
        d[i] = x[2 * i + 1];
      }
      wrow2::row_sync(sm.bar_id);
      wrow2::fwd<WI, OP, P0, HMAX, 0, EDGE>(s, d, buf, p.prog, p.levels, sm, p.bc);
    } else {
      constexpr int TOP = reg_max_levels(WI, OP, P0) - 1;
      wrow2::rev<WI, OP, P0, HMAX, TOP, EDGE>(s, d, buf, p.prog, p.levels, sm, p.bc);
      wrow2::row_sync(sm.bar_id);
      float x[2 * P0];
#pragma unroll
      for (int i = 0; i < P0; ++i) {
        x[2 * i] = s[i];
        x[2 * i + 1] = d[i];
      }
      wrow::write_run<float, 2 * P0, 2 * P0>(buf, 2 * P0 * g, x);
    }
    wrow2::row_sync(sm.bar_id);
    int64_t bin, bout;
    line_base(p.g, row, bin, bout);
    float* dst = p.out + bout;
#pragma unroll 4
    for (int u = t64; u < UNITS; u += 64) {
      const int sh = FWD ? wrow2::banded_shift(u, nbl) : SHA;
      st_hint(dst + (int64_t)u * 4, *reinterpret_cast<const float4*>(buf + wrow::swz(u, sh) * 4),
              pol_st);
    }
    wrow2::row_sync(sm.bar_id);  // buffer drained before a later copy refills it
    cur ^= 1;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

}  // namespace lw
