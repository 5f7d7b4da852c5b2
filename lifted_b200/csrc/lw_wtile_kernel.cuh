// Windowed warp-per-row kernel for long contiguous rows (rows too long for
// one warp's registers, e.g. 64 rows of 65536 float64): the levels of the
// pass run on windows of W = 64 * P0 samples, one warp per window.
//
// Window w of a row covers [wstart, wstart + W) with wstart = w * tile -
// halo; its interior [w * tile, (w + 1) * tile) is what it stores, of every
// detail band and of the last approximation band.  The halo (a multiple of
// 2 * P0) covers the samples that the window's edges corrupt over the
// levels, so interior values are those of the whole row.  Window starts and
// row lengths are multiples of 2 * P0, so at every level a lane's pairs lie
// wholly inside or wholly outside the row's band: a lane skips its
// neighbour's values when the neighbour is past a band edge (the Zero
// boundary's skipped taps) or past the window's edge (corrupted margins,
// never stored).
//
// Forward-stepping passes stage the raw window (coalesced 16-byte cp.async
// with zero fill outside the row), run the levels in registers exactly as
// the warp-per-row kernel does and assemble the window's bands in the same
// banded shared-memory layout; the interiors leave with coalesced stores.
// Reverse-stepping passes stage the window of every band in that layout,
// run the levels coarse to fine and store the interior of the rebuilt row.
#pragma once

#include <cstdint>

#include "lw_pdl.hpp"
#include "lw_wrow_kernel.cuh"

namespace lw {

template <typename T>
struct WTileParams {
  const T* in;
  T* out;
  LineGeom g;        // contiguous rows (g.sin == g.sout == 1)
  int64_t tile;      // interior samples per window (a multiple of 2 * P0)
  int64_t halo;      // samples per side (a multiple of 2 * P0)
  int64_t ntiles;    // windows per row
  int32_t levels;    // every level of the pass, in registers
  int32_t pad_;
  DevProgram<T> prog;
};

namespace wtile {

// Address of element e of a window buffer in the banded layout (bands of
// the window: a_L in [0, nbl), d_l in [W >> l, W >> (l - 1))).
template <typename T>
__device__ __forceinline__ T* banded(T* buf, int e, int nbl) {
  constexpr int EPU = 16 / (int)sizeof(T);
  const int u = e / EPU;
  return buf + wrow::swz(u, wrow::banded_shift<T>(u, nbl)) * EPU + (e % EPU);
}

// Stages window positions [w0, w0 + cnt) of a band (row positions
// [base, base + lim) of the line at src) into buffer elements [r, r + cnt)
// of the banded layout, zeros outside the band: 16-byte cp.async units with
// zero fill when the window start and the band are unit-aligned, else
// element by element.
template <typename T>
__device__ __forceinline__ void stage_band(T* buf, int nbl, int r, int cnt, const T* src,
                                           int64_t base, int64_t lim, int64_t w0, int lane) {
  constexpr int EPU = 16 / (int)sizeof(T);
  if ((w0 % EPU) == 0 && (lim % EPU) == 0 && (base % EPU) == 0 && (r % EPU) == 0 &&
      (cnt % EPU) == 0) {
    for (int j = lane * EPU; j < cnt; j += 32 * EPU) {
      const int64_t pos = w0 + j;
      const bool in_band = pos >= 0 && pos < lim;
      const unsigned saddr = (unsigned)__cvta_generic_to_shared(banded(buf, r + j, nbl));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr),
                   "l"(in_band ? src + base + pos : src), "r"(in_band ? 16 : 0)
                   : "memory");
    }
  } else {
    for (int j = lane; j < cnt; j += 32) {
      const int64_t pos = w0 + j;
      *banded(buf, r + j, nbl) = (pos >= 0 && pos < lim) ? src[base + pos] : T(0);
    }
  }
}

// Stores buffer elements [b0, b0 + cnt) of the banded layout to dst[0 ..
// cnt): 16-byte units when everything is unit-aligned, else elements.
template <typename T>
__device__ __forceinline__ void drain_band(T* dst, T* buf, int nbl, int b0, int cnt,
                                           int64_t dst_off, int lane) {
  constexpr int EPU = 16 / (int)sizeof(T);
  if ((b0 % EPU) == 0 && (cnt % EPU) == 0 && (dst_off % EPU) == 0) {
    for (int j = lane * EPU; j < cnt; j += 32 * EPU) {
      const int4 v = *reinterpret_cast<const int4*>(banded(buf, b0 + j, nbl));
      *reinterpret_cast<int4*>(dst + j) = v;
    }
  } else {
    for (int j = lane; j < cnt; j += 32) dst[j] = *banded(buf, b0 + j, nbl);
  }
}

template <typename T, int WI, int OP, int P0, int LV, bool EM>
__device__ __forceinline__ void fwd(T (&s)[P0], T (&d)[P0], T* buf, const DevProgram<T>& prog,
                                    int levels, int lane, int64_t wstart, int64_t n) {
  constexpr int P = P0 >> LV;
  if constexpr (P >= 1 && P >= kreach(WI, OP)) {
    if (LV < levels) {
      constexpr int NB = 32 * P;
      const int64_t nbp = n >> (LV + 1);                 // pairs of the row's band
      const int64_t gp0 = (wstart >> (LV + 1)) + (int64_t)lane * P;
      const int64_t rem = nbp - gp0;                     // the band ends in this lane
      const int lim = rem >= P ? P : (rem > 0 ? (int)rem : 0);
      const int rlim = rem - P >= P ? P : (rem - P > 0 ? (int)(rem - P) : 0);  // or the next
      wrow::wsteps<T, WI, OP, 0, P, P0, EM>(s, d, prog, lane > 0 && gp0 > 0,
                                            lane < 31 && gp0 + P < nbp, lim, rlim);
      wrow::write_run<T, P, P>(buf, NB + P * lane, d);
      if (LV + 1 == levels) {
        wrow::write_run<T, P, P>(buf, P * lane, s);
        return;
      }
#pragma unroll
      for (int i = 0; i < P / 2; ++i) {
        d[i] = s[2 * i + 1];
        s[i] = s[2 * i];
      }
      fwd<T, WI, OP, P0, LV + 1, EM>(s, d, buf, prog, levels, lane, wstart, n);
    }
  }
}

template <typename T, int WI, int OP, int P0, int LV, bool EM>
__device__ __forceinline__ void rev(T (&s)[P0], T (&d)[P0], T* buf, const DevProgram<T>& prog,
                                    int levels, int lane, int64_t wstart, int64_t n) {
  constexpr int P = P0 >> LV;
  if constexpr (LV >= 0) {
    if constexpr (P >= 1 && P >= kreach(WI, OP)) {
      if (LV < levels) {
        constexpr int NB = 32 * P;
        const int64_t nbp = n >> (LV + 1);
        const int64_t gp0 = (wstart >> (LV + 1)) + (int64_t)lane * P;
        const int64_t rem = nbp - gp0;
        const int lim = rem >= P ? P : (rem > 0 ? (int)rem : 0);
        const int rlim = rem - P >= P ? P : (rem - P > 0 ? (int)(rem - P) : 0);
        if (LV + 1 == levels) wrow::read_run<T, P, P>(buf, P * lane, s);
        wrow::read_run<T, P, P>(buf, NB + P * lane, d);
        wrow::wsteps<T, WI, OP, 0, P, P0, EM>(s, d, prog, lane > 0 && gp0 > 0,
                                              lane < 31 && gp0 + P < nbp, lim, rlim);
        if constexpr (LV > 0) {
#pragma unroll
          for (int i = P - 1; i >= 0; --i) {
            s[2 * i + 1] = d[i];
            s[2 * i] = s[i];
          }
        }
      }
    }
    if constexpr (LV > 0) rev<T, WI, OP, P0, LV - 1, EM>(s, d, buf, prog, levels, lane, wstart, n);
  }
}

}  // namespace wtile

// 128 threads = four windows, one warp each; no block barriers.
// EM: rows whose length is a multiple of 2^levels but not of 2 * P0 (the
// band ends inside a lane at some level).
template <typename T, int WI, int OP, int P0, bool EM>
__global__ void __launch_bounds__(128)
    wtile_kernel(const __grid_constant__ WTileParams<T> p) {
  constexpr int W = 64 * P0;                  // window samples
  constexpr int EPU = 16 / (int)sizeof(T);    // elements per 16-byte unit
  constexpr int UNITS = W / EPU;
  constexpr bool FWD = (OP == TF_F || OP == TF_IA);
  constexpr int SHA = wrow::swz_shift_bytes(2 * P0 * (int)sizeof(T));
  extern __shared__ __align__(16) unsigned char lw_wtile_smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t item = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (item >= p.g.nlines * p.ntiles) return;  // whole warps only
  pdl_wait();  // the previous kernel's results (no global access before)
  pdl_trigger();
  T* buf = reinterpret_cast<T*>(lw_wtile_smem) + (int64_t)warp * W;
  const int64_t row = item / p.ntiles;
  const int64_t w = item - row * p.ntiles;
  int64_t bin, bout;
  line_base(p.g, row, bin, bout);
  const int64_t n = p.g.n;
  const int64_t t0 = w * p.tile;
  const int64_t t1 = t0 + p.tile < n ? t0 + p.tile : n;
  const int64_t wstart = t0 - p.halo;
  const int L = p.levels;
  const int nbl = W >> L;

  T s[P0], d[P0];
  if constexpr (FWD) {
    // raw window, zeros outside the row (a unit across the row's end is
    // copied in part and zero-filled)
    const T* src = p.in + bin;
#pragma unroll 4
    for (int u = lane; u < UNITS; u += 32) {
      const int64_t e = wstart + (int64_t)u * EPU;
      const bool in_row = e >= 0 && e < n;
      const int bytes = !in_row ? 0 : (e + EPU <= n ? 16 : (int)((n - e) * (int64_t)sizeof(T)));
      const unsigned saddr = (unsigned)__cvta_generic_to_shared(buf + wrow::swz(u, SHA) * EPU);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr),
                   "l"(in_row ? src + e : src), "r"(bytes)
                   : "memory");
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
    T x[2 * P0];
    wrow::read_run<T, 2 * P0, 2 * P0>(buf, 2 * P0 * lane, x);
#pragma unroll
    for (int i = 0; i < P0; ++i) {
      s[i] = x[2 * i];
      d[i] = x[2 * i + 1];
    }
    __syncwarp();
    wtile::fwd<T, WI, OP, P0, 0, EM>(s, d, buf, p.prog, L, lane, wstart, n);
    __syncwarp();
    // interiors: d_l at out[n >> l + (t0 >> l) ..], a_L at out[t0 >> L ..]
    T* dst = p.out + bout;
    for (int l = 1; l <= L; ++l) {
      const int64_t o = (n >> l) + (t0 >> l);
      wtile::drain_band<T>(dst + o, buf, nbl, (W >> l) + (int)(p.halo >> l),
                           (int)((t1 - t0) >> l), o, lane);
    }
    wtile::drain_band<T>(dst + (t0 >> L), buf, nbl, (int)(p.halo >> L), (int)((t1 - t0) >> L),
                         t0 >> L, lane);
  } else {
    // the window of every band: a_L at in[wstart >> L ..], d_l at
    // in[n >> l + (wstart >> l) ..]; zeros outside the row's bands
    const T* src = p.in + bin;
    wtile::stage_band<T>(buf, nbl, 0, nbl, src, 0, n >> L, wstart >> L, lane);
    for (int l = 1; l <= L; ++l)
      wtile::stage_band<T>(buf, nbl, W >> l, W >> l, src, n >> l, n >> l, wstart >> l, lane);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
    constexpr int TOP = reg_max_levels(WI, OP, P0) - 1;
    wtile::rev<T, WI, OP, P0, TOP, EM>(s, d, buf, p.prog, L, lane, wstart, n);
    __syncwarp();
    T x[2 * P0];
#pragma unroll
    for (int i = 0; i < P0; ++i) {
      x[2 * i] = s[i];
      x[2 * i + 1] = d[i];
    }
    wrow::write_run<T, 2 * P0, 2 * P0>(buf, 2 * P0 * lane, x);
    __syncwarp();
    // interior [t0, t1): whole 16-byte units (halo and t0 are multiples of
    // 2 * P0; a row end inside a unit is stored element by element)
    T* o = p.out + bout + t0;
    const int u0 = (int)(p.halo / EPU);
    const int cnt = (int)((t1 - t0) / EPU);
    for (int j = lane; j < cnt; j += 32)
      *reinterpret_cast<int4*>(o + (int64_t)j * EPU) =
          *reinterpret_cast<const int4*>(buf + wrow::swz(u0 + j, SHA) * EPU);
    for (int e = cnt * EPU + lane; e < (int)(t1 - t0); e += 32) {
      const int b = (int)p.halo + e;
      o[e] = buf[wrow::swz(b / EPU, SHA) * EPU + (b % EPU)];
    }
  }
}

}  // namespace lw
