// Persistent TMA-staged kernel for strided axes (float32): the first k
// levels of an axis pass on windows of 512 samples x 32 adjacent lines.
//
// The lines of a strided axis pass are columns of a 2D (or 3D) view whose
// fastest dimension is contiguous: 32 adjacent lines give 128-byte rows.  A
// CTA (512 threads: lane = line, 16 chunks of 32 samples along the axis)
// loops over its tiles.  For each tile one thread issues TMA copies
// (cp.async.bulk.tensor with 2D/3D boxes, completion on an mbarrier) of the
// tile's rows into a 64 KiB staging buffer; every thread then moves its
// chunk from the staging buffer into registers, the CTA releases the buffer
// and the TMA engine fetches the next tile while the CTA lifts and stores
// the current one.  Forward-stepping passes stage the raw window (two boxes
// of 256 rows); reverse-stepping passes stage the window of every detail
// band d_1 .. d_k and of the approximation band a_k (one box each).
//
// The lifting arithmetic, the mailbox neighbour exchange and the band
// stores are those of the register-blocked kernel (lw_reg_kernel.cuh,
// tile mode): interior results are exact, the halo absorbs the corrupted
// window margins, out-of-band taps are skipped (Zero boundary).
#pragma once

#include <cuda.h>

#include <cstdint>

#include "lw_reg_kernel.cuh"

namespace lw {

constexpr int COL_P0 = 16;                             // pairs per chunk
constexpr int COL_LANES = 32;                          // lines per tile
constexpr int COL_CHUNKS = 16;                         // chunks per window
constexpr int COL_ROWS = 2 * COL_P0 * COL_CHUNKS;      // 512 window samples
constexpr int COL_THREADS = COL_LANES * COL_CHUNKS;    // 512
constexpr int COL_MAXK = 5;                            // levels per tile launch

struct ColParams {
  // tm_rows[i]: the input viewed as {lines (x), axis (y)[, outer (z)]},
  // box {32, 256 >> i[, 1]}; tm_tmp: the approximation band buffer
  // [position][line], box {32, 512 >> k}.
  CUtensorMap tm_rows[COL_MAXK];
  CUtensorMap tm_tmp;
  RegParams<float> r;   // geometry, program, tile, band buffer, levels
  int64_t ncols;        // lines along x (multiple of 32)
  int64_t nouter;       // z extent (1 for a 2D view)
  int64_t ntr;          // row tiles per strip
  int64_t ntiles;       // ncols/32 * ntr * nouter
  int32_t rank3;        // tensor maps are 3D
  int32_t a_from_tmp;   // reverse: a_k is in the band buffer (else in `in`)
  int32_t spin_limit;   // mbarrier polls before giving up
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

// TMA load of one box into shared memory (no multicast).
__device__ __forceinline__ void tma_box(void* dst, const CUtensorMap* tm, int x, int y,
                                        int z, bool rank3, uint64_t* bar) {
  if (rank3) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
  } else {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
  }
}

struct TileCoord {
  int64_t outer, col0, rt, wstart;
};

__device__ __forceinline__ TileCoord decode(const ColParams& p, int64_t t) {
  const int64_t nstrips = p.ncols / COL_LANES;
  const int64_t per_outer = nstrips * p.ntr;
  TileCoord c;
  c.outer = t / per_outer;
  const int64_t rem = t - c.outer * per_outer;
  const int64_t strip = rem / p.ntr;
  c.rt = rem - strip * p.ntr;
  c.col0 = strip * COL_LANES;
  c.wstart = c.rt * p.r.tile - p.r.halo;
  return c;
}

// Issues the TMA copies of tile t into the staging buffer (one thread).
template <bool FWD>
__device__ __forceinline__ void issue(const ColParams& p, int64_t t, float* stage,
                                      uint64_t* bar) {
  const TileCoord tc = decode(p, t);
  const int x = (int)tc.col0, z = (int)tc.outer;
  const bool r3 = p.rank3 != 0;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (FWD) {
    mbar_expect(bar, COL_ROWS * COL_LANES * sizeof(float));
    tma_box(stage, &p.tm_rows[0], x, (int)tc.wstart, z, r3, bar);
    tma_box(stage + 256 * COL_LANES, &p.tm_rows[0], x, (int)tc.wstart + 256, z, r3, bar);
  } else {
    // d_l windows at rows m_l + (wstart >> l), l = 1..k, then a_k
    const int k = p.r.nreg;
    mbar_expect(bar, COL_ROWS * COL_LANES * sizeof(float));
    int row = 0;
    for (int l = 1; l <= k; ++l) {
      const int64_t ml = p.r.g.n >> l;
      tma_box(stage + (size_t)row * COL_LANES, &p.tm_rows[l - 1], x,
              (int)(ml + (tc.wstart >> l)), z, r3, bar);
      row += COL_ROWS >> l;
    }
    if (p.a_from_tmp) {
      // band buffer: x = line index, y = position
      const int64_t L0 = tc.outer * p.ncols + tc.col0;
      tma_box(stage + (size_t)row * COL_LANES, &p.tm_tmp, (int)L0, (int)(tc.wstart >> k), 0,
              false, bar);
    } else {
      tma_box(stage + (size_t)row * COL_LANES, &p.tm_rows[k - 1], x, (int)(tc.wstart >> k), z,
              r3, bar);
    }
  }
}

// Reverse-stepping register levels with the detail values preloaded:
// dd[off(LV) + i] holds pair i of this chunk's d at level LV, where
// off(LV) = sum_{l < LV} (P0 >> l).
template <int LV, int P0>
constexpr int dd_off() {
  int o = 0;
  for (int l = 0; l < LV; ++l) o += P0 >> l;
  return o;
}

template <int WI, int OP, int P0, int HMAX, int LV>
__device__ __forceinline__ void rev_levels_pre(float (&s)[P0], float (&d)[P0],
                                               const float (&dd)[2 * P0], reg::Ctx<float>& c) {
  constexpr int P = P0 >> LV;
  if constexpr (LV >= 0) {
    if constexpr (P >= 1 && P >= cat_reach(WI, OP)) {
      if (LV < c.p->nreg) {
        const RegParams<float>& p = *c.p;
        const int64_t nb = c.n >> (LV + 1);
        const int64_t gp0 = c.e0 >> (LV + 1);
#pragma unroll
        for (int i = 0; i < P; ++i) d[i] = dd[dd_off<LV, P0>() + i];
        reg::steps<float, float, WI, OP, 0, P, P0, HMAX>(s, d, c, gp0, nb);
        if constexpr (LV == 0) {
          if (reg::chunk_stored(c)) {
            float* o = p.out + c.bout + c.e0 * p.g.sout;
#pragma unroll
            for (int i = 0; i < P; ++i) {
              o[(2 * i) * p.g.sout] = s[i];
              o[(2 * i + 1) * p.g.sout] = d[i];
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
      if constexpr (LV > 0) rev_levels_pre<WI, OP, P0, HMAX, LV - 1>(s, d, dd, c);
    } else if constexpr (LV > 0) {
      rev_levels_pre<WI, OP, P0, HMAX, LV - 1>(s, d, dd, c);
    }
  }
}

}  // namespace col

template <int WI, int OP>
__global__ void __launch_bounds__(COL_THREADS, 1)
    col_kernel(const __grid_constant__ ColParams p) {
  constexpr int P0 = COL_P0;
  constexpr int HMAX = cat_reach(WI, OP) > 0 ? cat_reach(WI, OP) : 1;
  constexpr bool FWD = (OP == TF_F || OP == TF_IA);
  extern __shared__ __align__(128) unsigned char col_smem[];
  float* stage = reinterpret_cast<float*>(col_smem);
  float* mbox = stage + COL_ROWS * COL_LANES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(mbox + 4 * HMAX * COL_THREADS);

  const int tid = threadIdx.x;
  reg::Ctx<float> c;
  c.p = &p.r;
  c.nth = COL_THREADS;
  c.tid = tid;
  c.mb = mbox;
  c.cA = nullptr;
  c.cB = nullptr;
  c.j = tid % COL_LANES;
  c.r = tid / COL_LANES;
  c.tid_l = tid - COL_LANES;
  c.tid_r = tid + COL_LANES;
  c.has_l = c.r > 0;
  c.has_r = c.r < COL_CHUNKS - 1;
  c.n = p.r.g.n;

  if (tid == 0) col::mbar_init(bar);
  __syncthreads();
  uint32_t parity = 0;
  int64_t t = blockIdx.x;
  if (t < p.ntiles && tid == 0) col::issue<FWD>(p, t, stage, bar);
  for (; t < p.ntiles; t += gridDim.x) {
    const bool got = col::mbar_wait(bar, parity, p.spin_limit);
    if (!__syncthreads_and(got)) {
      if (tid == 0) atomicExch(p.err, 1);
      col::mbar_wait(bar, parity, p.spin_limit);  // let a late copy land
      return;
    }
    parity ^= 1;
    const col::TileCoord tc = col::decode(p, t);
    const int64_t L = tc.outer * p.ncols + tc.col0 + c.j;
    c.L = L;
    c.line_ok = L < p.r.g.nlines;
    c.bin = 0;
    c.bout = 0;
    if (c.line_ok) line_base(p.r.g, L, c.bin, c.bout);
    c.buf = 0;
    c.e0 = tc.wstart + (int64_t)2 * P0 * c.r;
    c.tile_lo = tc.rt * p.r.tile;
    c.tile_hi = c.tile_lo + p.r.tile < c.n ? c.tile_lo + p.r.tile : c.n;

    float s[P0], d[P0];
    float dd[2 * P0];
    if constexpr (FWD) {
      const float* st = stage + (size_t)(c.r * 2 * P0) * COL_LANES + c.j;
#pragma unroll
      for (int i = 0; i < P0; ++i) {
        s[i] = st[(2 * i) * COL_LANES];
        d[i] = st[(2 * i + 1) * COL_LANES];
      }
    } else {
      const int k = p.r.nreg;
      int row = 0;
#pragma unroll
      for (int lv = 0; lv < COL_MAXK; ++lv) {
        if (lv < k) {
          const int P = P0 >> lv;
          const float* st = stage + (size_t)(row + c.r * P) * COL_LANES + c.j;
          const int off = (2 * P0) - (2 * P0 >> lv);  // sum_{l<lv} P0 >> l
#pragma unroll
          for (int i = 0; i < (P0 >> lv); ++i) dd[off + i] = st[i * COL_LANES];
          row += COL_ROWS >> (lv + 1);
        }
      }
      const int Pa = P0 >> (k - 1);
      const float* st = stage + (size_t)(row + c.r * Pa) * COL_LANES + c.j;
#pragma unroll
      for (int i = 0; i < P0; ++i)
        if (i < Pa) s[i] = st[i * COL_LANES];
    }
    __syncthreads();  // staging consumed
    if (tid == 0 && t + gridDim.x < p.ntiles) col::issue<FWD>(p, t + gridDim.x, stage, bar);

    if constexpr (FWD) {
      reg::fwd_levels<float, float, 1, WI, OP, P0, HMAX, 0, true>(s, d, c);
    } else {
      constexpr int TOP = reg_max_levels(WI, OP, P0) - 1;
      col::rev_levels_pre<WI, OP, P0, HMAX, TOP>(s, d, dd, c);
    }
  }
}

}  // namespace lw
