// Persistent TMA-staged kernel for strided axes (float32, float64): the first k
// levels of an axis pass on windows of 512 samples x 32*V adjacent lines.
//
// The lines of a strided axis pass are columns of a 2D (or 3D) view whose
// fastest dimension is contiguous: 32*V adjacent lines give 128*V-byte rows.
// A CTA (512 threads: lane = V adjacent lines, 16 chunks of 32 samples along
// the axis) loops over its tiles.  For each tile one thread issues TMA
// copies (cp.async.bulk.tensor with 2D/3D boxes, completion on an mbarrier)
// of the tile's rows into the staging buffer; the threads move their chunks
// into registers, the CTA releases the buffer and the TMA engine fetches the
// next tile while the CTA lifts and stores the current one.
//
//   forward-stepping  stages the raw window (two boxes of 256 rows); every
//                     thread takes its whole chunk, then the buffer is free;
//   reverse-stepping  stages the window of every detail band d_1 .. d_k and
//                     of the approximation band a_k (one box each); threads
//                     take d_1 at once and read the coarser bands level by
//                     level, and the buffer is released after the last of
//                     those reads (level 2), so the next tile's copy overlaps
//                     the two finest levels.
//
// With V = 2 (float32) a lane holds two adjacent lines and every step runs on
// packed FP32x2 arithmetic (lw_reg_kernel.cuh, LaneVec), halving the
// instructions.  float64 runs with V = 1 and reads d_1 from the staging
// buffer at the finest level (its registers hold no preloaded copy), so its
// reverse passes release the buffer one level later.
// The lifting arithmetic, the mailbox neighbour exchange and the band
// stores are those of the register-blocked kernel in tile mode: interior
// results are exact, the halo absorbs the corrupted window margins,
// out-of-band taps are skipped (Zero boundary; the EDGE instantiation redoes
// the band edges of the Constant, Symmetric and Reflect boundaries).
#pragma once

#include <cuda.h>

#include <cstdint>

#include "lw_pdl.hpp"
#include "lw_reg_kernel.cuh"

namespace lw {

constexpr int COL_P0 = 16;                             // pairs per chunk
constexpr int COL_LANES = 32;                          // lanes per row
constexpr int COL_CHUNKS = 16;                         // chunks per window
constexpr int COL_ROWS = 2 * COL_P0 * COL_CHUNKS;      // 512 window samples
constexpr int COL_THREADS = COL_LANES * COL_CHUNKS;    // 512
constexpr int COL_MAXK = 5;                            // levels per tile launch

// Mailbox buffers of an instantiation: float64 with the wide generic
// exchange keeps one (its staging buffer and a double-buffered mailbox do
// not fit shared memory together), at the price of a second barrier per
// step; every other instantiation alternates two.
template <typename T, int WI>
constexpr int col_mb_bufs() {
  return (sizeof(T) == 8 && WI == WI_GENW) ? 1 : 2;
}

template <typename T>
struct ColParams {
  // tm_rows[i]: the input viewed as {lines (x), axis (y)[, outer (z)]},
  // box {32*V, 256 >> i[, 1]}; tm_tmp: the approximation band buffer
  // [position][line], box {32*V, 512 >> k}.
  CUtensorMap tm_rows[COL_MAXK];
  CUtensorMap tm_tmp;
  RegParams<T> r;       // geometry, program, tile, band buffer, levels
  int64_t ncols;        // lines along x (the last strip may be partial)
  int64_t nouter;       // z extent (1 for a 2D view)
  int64_t ntr;          // row tiles per strip
  int64_t ntiles;       // ceil(ncols/(32*V)) * ntr * nouter
  int32_t rank3;        // tensor maps are 3D
  int32_t a_from_tmp;   // reverse: a_k is in the band buffer (else in `in`)
  int32_t spin_limit;   // mbarrier polls before giving up
  int32_t stack;        // whole lines of 512/stack samples: a tile stacks
                        // `stack` consecutive outer slices (1: off)
  int32_t row_order;    // tiles numbered row tile major: CTAs that run at
                        // the same time read neighbouring strips of the
                        // same rows (else strip major)
  int32_t pad_;
  int32_t* err;         // set to 1 when a staging wait gave up
};

namespace col {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait for phase `parity` of the barrier.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// TMA load of one box into shared memory (no multicast), with an L2 cache
// policy.
__device__ __forceinline__ void tma_box(void* dst, const CUtensorMap* tm, int x, int y,
                                        int z, bool rank3, uint64_t* bar, uint64_t pol) {
  if (rank3) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        ".L2::cache_hint [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
  } else {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        ".L2::cache_hint [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
  }
}

struct TileCoord {
  int64_t outer, col0, rt, wstart;
};

template <typename T, int V>
__device__ __forceinline__ TileCoord decode(const ColParams<T>& p, int64_t t) {
  const int64_t nstrips = (p.ncols + COL_LANES * V - 1) / (COL_LANES * V);
  const int64_t per_outer = nstrips * p.ntr;
  TileCoord c;
  c.outer = t / per_outer;
  const int64_t rem = t - c.outer * per_outer;
  int64_t strip;
  if (p.row_order) {
    c.rt = rem / nstrips;
    strip = rem - c.rt * nstrips;
  } else {
    strip = rem / p.ntr;
    c.rt = rem - strip * p.ntr;
  }
  c.col0 = strip * COL_LANES * V;
  c.wstart = c.rt * p.r.tile - p.r.halo;
  c.outer *= p.stack;  // first slice of the tile's group
  return c;
}

// Issues the TMA copies of tile t into the staging buffer (one thread).
template <typename T, bool FWD, int V>
__device__ __forceinline__ void issue(const ColParams<T>& p, int64_t t, T* stage,
                                      uint64_t* bar) {
  constexpr int W = COL_LANES * V;  // elements per staging row
  const uint64_t pol = l2_load_policy(p.r.l2hint);
  const TileCoord tc = decode<T, V>(p, t);
  const int x = (int)tc.col0, z = (int)tc.outer;
  const bool r3 = p.rank3 != 0;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect(bar, COL_ROWS * W * sizeof(T));
  if (FWD) {
    // stacked: slices z .. z+stack-1 of n rows each, two boxes of half the
    // slices (256 rows each)
    const bool st = p.stack > 1;
    tma_box(stage, &p.tm_rows[0], x, (int)tc.wstart, z, r3, bar, pol);
    tma_box(stage + 256 * W, &p.tm_rows[0], x, st ? 0 : (int)tc.wstart + 256,
            st ? z + p.stack / 2 : z, r3, bar, pol);
  } else {
    // d_l windows at rows m_l + (wstart >> l), l = 1..k, then a_k
    const int k = p.r.nreg;
    int row = 0;
    for (int l = 1; l <= k; ++l) {
      // d_l starts at ceil(n / 2^l)
      const int64_t ml = (p.r.g.n + ((int64_t)1 << l) - 1) >> l;
      tma_box(stage + (size_t)row * W, &p.tm_rows[l - 1], x, (int)(ml + (tc.wstart >> l)), z,
              r3, bar, pol);
      row += COL_ROWS >> l;
    }
    if (p.a_from_tmp && p.stack > 1) {
      // band buffer viewed as {lines of a slice, position, slice}
      tma_box(stage + (size_t)row * W, &p.tm_tmp, x, 0, z, true, bar, pol);
    } else if (p.a_from_tmp) {
      // band buffer: x = line index, y = position
      const int64_t L0 = tc.outer * p.ncols + tc.col0;
      tma_box(stage + (size_t)row * W, &p.tm_tmp, (int)L0, (int)(tc.wstart >> k), 0, false, bar, pol);
    } else {
      tma_box(stage + (size_t)row * W, &p.tm_rows[k - 1], x, (int)(tc.wstart >> k), z, r3, bar, pol);
    }
  }
}

// One box of `rows` rows of 32 lanes from src (x along lines at unit stride,
// y at stride ystr, extents xdim and ydim) into dst, zeros outside the
// extents as the TMA's fill gives them; every thread of the CTA takes part.
template <typename T>
__device__ __forceinline__ void ld_box(T* dst, const T* src, int64_t xdim, int64_t ydim,
                                       int64_t ystr, int64_t x, int64_t y, int rows) {
  for (int e = threadIdx.x; e < rows * COL_LANES; e += COL_THREADS) {
    const int yi = e / COL_LANES, xi = e % COL_LANES;
    const int64_t xx = x + xi, yy = y + yi;
    dst[e] = (xx < xdim && yy >= 0 && yy < ydim) ? src[xx + yy * ystr] : T(0);
  }
}

// Plain-load form of issue() for lines whose stride (or line count, or
// base) TMA cannot take (strides and the band buffer's boxes must be
// multiples of 16 bytes): the same boxes, loaded by every thread with
// bounds checks; one line per lane, no stacked slices.
template <typename T, bool FWD>
__device__ __forceinline__ void fill(const ColParams<T>& p, int64_t t, T* stage) {
  const TileCoord tc = decode<T, 1>(p, t);
  const LineGeom& g = p.r.g;
  const int64_t x = tc.col0;
  const int64_t n = g.n;
  const bool zin = tc.outer < p.nouter;  // a z past the extent reads zeros
  const T* in = p.r.in + (g.nother == 2 ? tc.outer * g.oin[1] : 0);
  const int64_t xdim = zin ? p.ncols : 0;
  if (FWD) {
    ld_box(stage, in, xdim, n, g.sin, x, tc.wstart, COL_ROWS);
  } else {
    const int k = p.r.nreg;
    int row = 0;
    for (int l = 1; l <= k; ++l) {
      const int64_t ml = (n + ((int64_t)1 << l) - 1) >> l;
      ld_box(stage + (size_t)row * COL_LANES, in, xdim, n, g.sin, x, ml + (tc.wstart >> l),
             COL_ROWS >> l);
      row += COL_ROWS >> l;
    }
    if (p.a_from_tmp) {
      // band buffer [position][line] of ceil(n / 2^k) positions
      const int64_t m = (n + ((int64_t)1 << k) - 1) >> k;
      ld_box(stage + (size_t)row * COL_LANES, p.r.tmp, zin ? g.nlines : 0, m, g.nlines,
             tc.outer * p.ncols + x, tc.wstart >> k, COL_ROWS >> k);
    } else {
      ld_box(stage + (size_t)row * COL_LANES, in, xdim, n, g.sin, x, tc.wstart >> k,
             COL_ROWS >> k);
    }
  }
}

// Per-tile state of the reverse levels: where the staged bands are and how
// to hand the buffer back.
template <typename T>
struct RevStage {
  const T* stage;
  uint64_t* bar;
  const ColParams<T>* p;
  int64_t next;  // next tile of this CTA (>= ntiles: none)
  bool prefetch; // issue the next tile's copies once the buffer is free
};

// Staging row of pair 0 of this chunk in the band region of level LV
// (detail bands d_1.., region sizes 256, 128, ...) or of a_k (LV = k - 1).
__device__ __forceinline__ int region_row(int lv) { return COL_ROWS - (COL_ROWS >> lv); }

template <typename T, typename VT, int V, int P, int PA>
__device__ __forceinline__ void read_rows(VT (&v)[PA], const T* stage, int row0, int lane) {
  constexpr int W = COL_LANES * V;
  const T* q = stage + (size_t)row0 * W + lane * V;
#pragma unroll
  for (int i = 0; i < P; ++i) v[i] = *reinterpret_cast<const VT*>(q + (size_t)i * W);
}

// Whether the reverse levels keep d_1 in registers from the start (float32)
// or read it from the staging buffer at the finest level (float64, whose
// registers hold no room for the copy).
template <typename T>
constexpr bool preload_d1() {
  return sizeof(T) == 4;
}

template <typename T, int WI, int OP, int P0, int HMAX, int V, int LV, bool EM, bool EDGE>
__device__ __forceinline__ void rev_levels(typename LaneVec<T, V>::type (&s)[P0],
                                           typename LaneVec<T, V>::type (&d)[P0],
                                           const typename LaneVec<T, V>::type (&d1)[P0],
                                           reg::Ctx<T>& c, const RevStage<T>& rs) {
  using VT = typename LaneVec<T, V>::type;
  constexpr int P = P0 >> LV;
  // the level after whose reads the staging buffer is free
  constexpr int LAST_READ = preload_d1<T>() ? 1 : 0;
  if constexpr (LV >= 0) {
    if constexpr (P >= 1 && P >= kreach(WI, OP)) {
      const int k = c.p->nreg;
      if (LV < k) {
        const RegParams<T>& p = *c.p;
        const int64_t nb = c.n >> (LV + 1);
        const int64_t gp0 = c.e0 >> (LV + 1);
        if constexpr (EM) reg::level_lengths(c, LV);
        if (LV + 1 == k && (LV > 0 || !preload_d1<T>()))
          read_rows<T, VT, V, P, P0>(s, rs.stage, region_row(k) + c.r * P, c.j);
        if constexpr (LV > 0 || !preload_d1<T>()) {
          read_rows<T, VT, V, P, P0>(d, rs.stage, region_row(LV) + c.r * P, c.j);
        } else {
#pragma unroll
          for (int i = 0; i < P0; ++i) d[i] = d1[i];
        }
        if (LV == LAST_READ) {
          // last read of the staging buffer for this tile
          __syncthreads();
          if (c.tid == 0 && rs.prefetch && rs.next < rs.p->ntiles)
            issue<T, false, V>(*rs.p, rs.next, const_cast<T*>(rs.stage), rs.bar);
        }
        reg::steps_sel<T, VT, WI, OP, P, P0, HMAX, EM, EDGE>(s, d, c, gp0, nb);
        if constexpr (LV == 0) {
          if (reg::chunk_stored(c)) {
            T* o = p.out + c.bout + c.e0 * p.g.sout;
            // EM: the line may end inside this chunk, after an s value
            // (odd length)
            const int lim_s = !EM ? P : reg::chunk_lim(c.nsl, gp0, P);
            const int lim_d = !EM ? P : reg::chunk_lim(c.ndl, gp0, P);
#pragma unroll
            for (int i = 0; i < P; ++i) {
              if (!EM || i < lim_s) st_hint(o + (2 * i) * p.g.sout, s[i], c.pol_st);
              if (!EM || i < lim_d) st_hint(o + (2 * i + 1) * p.g.sout, d[i], c.pol_st);
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
      if constexpr (LV > 0) rev_levels<T, WI, OP, P0, HMAX, V, LV - 1, EM, EDGE>(s, d, d1, c, rs);
    } else if constexpr (LV > 0) {
      rev_levels<T, WI, OP, P0, HMAX, V, LV - 1, EM, EDGE>(s, d, d1, c, rs);
    }
  }
}

}  // namespace col

// EM: lines whose length is a multiple of 2^levels but not of 32 (the band
// ends inside a chunk at some level; taps and stores past it are skipped).
// EDGE: the instantiation for the Constant, Symmetric and Reflect
// boundaries (exact band edges, lw_edge.cuh); Zero passes run the one
// without that code.
// LDG: tiles staged by plain loads (col::fill) instead of TMA, for strides
// TMA cannot take; no copy of the next tile runs during the levels.
template <typename T, int WI, int OP, int V, bool EM, bool EDGE = false, bool LDG = false>
__global__ void __launch_bounds__(COL_THREADS, 1)
    col_kernel(const __grid_constant__ ColParams<T> p) {
  using VT = typename LaneVec<T, V>::type;
  static_assert(V == 1 || sizeof(T) == 4, "packed lanes are float32 only");
  static_assert(!LDG || V == 1, "plain-load staging takes one line per lane");
  constexpr int P0 = COL_P0;
  constexpr int W = COL_LANES * V;
  constexpr int HMAX = khmax(WI, OP);
  constexpr bool FWD = (OP == TF_F || OP == TF_IA);
  extern __shared__ __align__(128) unsigned char col_smem[];
  T* stage = reinterpret_cast<T*>(col_smem);
  T* mbox = stage + COL_ROWS * W;
  constexpr int MBB = col_mb_bufs<T, WI>();
  uint64_t* bar = reinterpret_cast<uint64_t*>(mbox + 2 * MBB * HMAX * COL_THREADS * V);

  const int tid = threadIdx.x;
  reg::Ctx<T> c;
  c.p = &p.r;
  c.nth = COL_THREADS;
  c.tid = tid;
  c.mb = mbox;
  c.cA = nullptr;
  c.cB = nullptr;
  c.mb_bufs = MBB;
  c.j = tid % COL_LANES;
  c.r = tid / COL_LANES;
  c.tid_l = tid - COL_LANES;
  c.tid_r = tid + COL_LANES;
  c.has_l = c.r > 0;
  c.has_r = c.r < COL_CHUNKS - 1;
  c.n = p.r.g.n;
  c.bc = p.r.bc;
  c.pol_st = l2_store_policy(p.r.l2hint);
  // stacked tiles: chunk r holds chunk rr of slice zr (its own line, whose
  // band edges mask the taps that would reach the neighbouring slices)
  const int cps = p.stack > 1 ? (int)(c.n / (2 * P0)) : COL_CHUNKS;
  const int zr = c.r / cps;
  const int rr = c.r - zr * cps;

  if (tid == 0) col::mbar_init(bar);
  __syncthreads();
  pdl_wait();  // the previous kernel's results (no global access before)
  uint32_t parity = 0;
  int64_t t = blockIdx.x;
  if (!LDG && t < p.ntiles && tid == 0) col::issue<T, FWD, V>(p, t, stage, bar);
  for (; t < p.ntiles; t += gridDim.x) {
    if (t + gridDim.x >= p.ntiles) pdl_trigger();  // the CTA's last tile
    if constexpr (LDG) {
      // the previous tile's last staging read precedes a block barrier
      col::fill<T, FWD>(p, t, stage);
      __syncthreads();
    } else {
    const bool got = col::mbar_wait(bar, parity, p.spin_limit);
    if (!__syncthreads_and(got)) {
      // Give up on the tile (the host reads the flag), but do not leave
      // while the tile's copy may still be writing this CTA's shared memory,
      // which the SM hands to the next CTA once this one exits: the copy
      // of tile t is the only one in flight here (the next tile's copy is
      // issued after this wait), so wait for it to land, bounded again but
      // sixteen times longer.  Only a copy that never completes at all gets
      // past this second bound.
      if (tid == 0) atomicExch(p.err, 1);
      col::mbar_wait(bar, parity, 16 * p.spin_limit);  // the host caps spin_limit at 2^22
      __syncthreads();
      return;
    }
    parity ^= 1;
    }
    const col::TileCoord tc = col::decode<T, V>(p, t);
    const int64_t outer = tc.outer + zr;
    const int64_t L = outer * p.ncols + tc.col0 + (int64_t)c.j * V;
    c.L = L;
    // V lines together; the last strip of a slice may run past ncols (its
    // lanes there hold the TMA's zero fill and store nothing), and a last
    // group of stacked slices past the outer extent
    c.line_ok = outer < p.nouter && tc.col0 + (int64_t)(c.j + 1) * V <= p.ncols &&
                L < p.r.g.nlines;
    c.bin = 0;
    c.bout = 0;
    if (c.line_ok) line_base(p.r.g, L, c.bin, c.bout);
    c.buf = 0;
    c.e0 = tc.wstart + (int64_t)2 * P0 * rr;
    c.tile_lo = tc.rt * p.r.tile;
    c.tile_hi = c.tile_lo + p.r.tile < c.n ? c.tile_lo + p.r.tile : c.n;
    const int64_t next = t + gridDim.x;

    VT s[P0], d[P0];
    if constexpr (FWD) {
      const T* st = stage + (size_t)(c.r * 2 * P0) * W + c.j * V;
#pragma unroll
      for (int i = 0; i < P0; ++i) {
        s[i] = *reinterpret_cast<const VT*>(st + (size_t)(2 * i) * W);
        d[i] = *reinterpret_cast<const VT*>(st + (size_t)(2 * i + 1) * W);
      }
      __syncthreads();  // staging consumed
      if (!LDG && tid == 0 && next < p.ntiles) col::issue<T, FWD, V>(p, next, stage, bar);
      reg::fwd_levels<T, VT, V, WI, OP, P0, HMAX, 0, true, EM, EDGE>(s, d, c);
    } else {
      const int k = p.r.nreg;
      VT d1[col::preload_d1<T>() ? P0 : 1];
      if constexpr (col::preload_d1<T>()) {
        col::read_rows<T, VT, V, P0, P0>(d1, stage, c.r * P0, c.j);  // d_1 region
        if (k == 1) {
          col::read_rows<T, VT, V, P0, P0>(s, stage, col::region_row(1) + c.r * P0, c.j);
          __syncthreads();
          if (!LDG && tid == 0 && next < p.ntiles) col::issue<T, FWD, V>(p, next, stage, bar);
        }
      }
      col::RevStage<T> rs{stage, bar, &p, next, !LDG};
      constexpr int TOP = reg_max_levels(WI, OP, P0) - 1;
      if constexpr (col::preload_d1<T>()) {
        col::rev_levels<T, WI, OP, P0, HMAX, V, TOP, EM, EDGE>(s, d, d1, c, rs);
      } else {
        VT dummy[P0];
        col::rev_levels<T, WI, OP, P0, HMAX, V, TOP, EM, EDGE>(s, d, dummy, c, rs);
      }
    }
  }
}

}  // namespace lw
