// Warp-per-row lifting kernel of the B200 DWT (fast path for contiguous rows
// of 64 * P0 elements).
//
// One warp owns one whole row: lane l holds pairs [P0*l, P0*l + P0) of level
// 1 in registers, and every level of the row runs in those registers.  The
// neighbour values a lifting step needs cross between lanes by warp shuffles,
// so the kernel has no block barriers at all; the split of a level's
// approximation band into the next level's pairs is a register renaming.
//
// The row moves through shared memory on both sides: a coalesced cp.async
// copy (16 bytes per lane, consecutive lanes on consecutive addresses) fills
// the warp's row buffer, each lane then reads its own contiguous chunk, and
// the detail bands of every level plus the final approximation are assembled
// in the same buffer and leave with coalesced 16-byte stores.  The buffer is
// XOR-swizzled in 16-byte units so that both the coalesced pass and the
// per-lane chunk pass are free of bank conflicts:
//   unit U (16 bytes) of the row lives at unit (U & ~7) | ((U ^ swz(U>>3)) & 7)
//   with swz(R) = (R >> log2(max(1, P0/16))) & 7.
//
// Arithmetic per element is the reference's Across form (see
// lw_reg_kernel.cuh); this kernel serves the Zero boundary, where the lanes
// at the row ends skip their out-of-band taps.
#pragma once

#include <cstdint>

#include "lw_edge.cuh"
#include "lw_reg_kernel.cuh"

namespace lw {

template <typename T>
struct WRowParams {
  const T* in;
  T* out;
  LineGeom g;        // contiguous rows (g.sin == g.sout == 1)
  int32_t levels;      // levels of the pass
  int32_t reg_levels;  // generic instantiation: levels in registers (the
                       // rest on compacted lanes); unused otherwise
  int32_t l2hint;      // two-warp kernel: L2 priorities (lw_cache.cuh)
  int32_t bc;          // boundary: Zero, or Constant / Symmetric / Reflect
                       // in the warp-per-row kernel's EDGE instantiation
  DevProgram<T> prog;
};

namespace wrow {

constexpr unsigned FULL = 0xffffffffu;

// XOR swizzle of 16-byte units for a buffer whose lanes each own a
// contiguous run of CHUNK elements: unit U of 128-byte row R = U >> 3 lives
// at (U & ~7) | ((U ^ (R >> SH)) & 7), SH = log2 of the 128-byte rows per
// lane run (0 when a run is shorter than a row).  Eight consecutive lanes
// then hit eight distinct 16-byte bank groups both when each lane walks its
// own run and when consecutive lanes take consecutive units.
constexpr int swz_shift_bytes(int bytes) {
  return bytes >= 1024 ? 3 : bytes >= 512 ? 2 : bytes >= 256 ? 1 : 0;
}

__device__ __forceinline__ int swz(int U, int sh) {
  const int R = U >> 3;
  return (U & ~7) | ((U ^ (R >> sh)) & 7);
}

// Layout of a row read (or written) as runs of CHUNK elements per lane.
template <typename T, int CHUNK>
__device__ __forceinline__ T* elem(T* buf, int e) {
  constexpr int EPU = 16 / (int)sizeof(T);
  constexpr int SH = swz_shift_bytes(CHUNK * (int)sizeof(T));
  return buf + swz(e / EPU, SH) * EPU + (e % EPU);
}

// Banded layout: the approximation [0, nbl) has runs of nbl/32 elements per
// lane, each detail band [2^k, 2^(k+1)) runs of 2^k/32.  Shift of unit U.
template <typename T>
__device__ __forceinline__ int banded_shift(int U, int nbl) {
  constexpr int EPU = 16 / (int)sizeof(T);
  const int e = U * EPU;
  const int region = e < nbl ? nbl : (1 << (31 - __clz(e)));
  const int bytes = (region / 32) * (int)sizeof(T);
  return bytes >= 1024 ? 3 : bytes >= 512 ? 2 : bytes >= 256 ? 1 : 0;
}

// Reads N consecutive elements starting at e (e aligned to min(N, EPU)).
template <typename T, int CHUNK, int N, int PA>
__device__ __forceinline__ void read_run(T* buf, int e, T (&v)[PA]) {
  constexpr int EPU = 16 / (int)sizeof(T);
  if constexpr (N >= EPU) {
#pragma unroll
    for (int i = 0; i < N; i += EPU) {
      const T* p = elem<T, CHUNK>(buf, e + i);
      if constexpr (sizeof(T) == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        v[i] = q.x; v[i + 1] = q.y; v[i + 2] = q.z; v[i + 3] = q.w;
      } else {
        const double2 q = *reinterpret_cast<const double2*>(p);
        v[i] = q.x; v[i + 1] = q.y;
      }
    }
  } else if constexpr (N == 2 && sizeof(T) == 4) {
    const float2 q = *reinterpret_cast<const float2*>(elem<T, CHUNK>(buf, e));
    v[0] = q.x; v[1] = q.y;
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = *elem<T, CHUNK>(buf, e + i);
  }
}

template <typename T, int CHUNK, int N, int PA>
__device__ __forceinline__ void write_run(T* buf, int e, const T (&v)[PA]) {
  constexpr int EPU = 16 / (int)sizeof(T);
  if constexpr (N >= EPU) {
#pragma unroll
    for (int i = 0; i < N; i += EPU) {
      T* p = elem<T, CHUNK>(buf, e + i);
      if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      } else {
        *reinterpret_cast<double2*>(p) = make_double2(v[i], v[i + 1]);
      }
    }
  } else if constexpr (N == 2 && sizeof(T) == 4) {
    *reinterpret_cast<float2*>(elem<T, CHUNK>(buf, e)) = make_float2(v[0], v[1]);
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) *elem<T, CHUNK>(buf, e + i) = v[i];
  }
}

// What a lane at a band end needs for the exact edges of the Constant,
// Symmetric and Reflect boundaries (lw_edge.cuh): the program, the
// boundary and the band's length in pairs.
template <typename T>
struct WEdge {
  const DevProgram<T>* prog;
  int bc;
  int64_t nb;
};

// One step over the lane's P pairs; halos by shuffle.  okl / okr: the
// left / right neighbour lane holds pairs of the same band (whole rows:
// lane > 0 / lane < the last active lane; windows: also by band position).
// EM: the band may end inside this lane, after its first `lim` pairs, or
// inside its right neighbour, after that lane's first `rlim` pairs (windows
// of rows whose length is not a multiple of the lane's pairs); taps past
// the end are skipped like taps past the band edge.
// EDGE: whole rows only (okl false exactly at the band's first lane, okr
// false at its last); the lanes at the band ends redo their edge around the
// Zero update when the boundary is not Zero (ed).
template <typename T, int P, int PA, int KIND, int OFF, int NT, int SUB,
          int HL, int HR, bool EM = false, bool EDGE = false>
__device__ __forceinline__ void wupdate(T (&y)[PA], const T (&x)[PA],
                                        const DevStep<T>& st, bool okl, bool okr,
                                        int lim = P, int rlim = P,
                                        const WEdge<T>* ed = nullptr) {
  static_assert(HL <= P && HR <= P, "step reaches past the neighbour lane");
  T xl[HL > 0 ? HL : 1], xr[HR > 0 ? HR : 1];
#pragma unroll
  for (int h = 0; h < HL; ++h) xl[h] = __shfl_up_sync(FULL, x[P - HL + h], 1);
#pragma unroll
  for (int h = 0; h < HR; ++h) xr[h] = __shfl_down_sync(FULL, x[h], 1);
  constexpr int E = P < edge::kEdge ? P : edge::kEdge;
  T sf[HL > 0 ? HL : 1], sb[HR > 0 ? HR : 1];
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
    T yi = y[i];
    if constexpr (KIND == K_GEN) {
#pragma unroll
      for (int k = 0; k < NT; ++k) {
        const int idx = i + OFF + k;
        const T v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
        const bool ok = idx < 0 ? okl : (idx >= P ? (okr && (!EM || idx - P < rlim)) : (!EM || idx < lim));
        const T f = fop(SUB, st.c[k], v, yi);
        yi = ok ? f : yi;
      }
    } else if constexpr (KIND == K_REPEAT) {
      int idx = i + OFF;
      T v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
      bool ok = idx < 0 ? okl : (idx >= P ? (okr && (!EM || idx - P < rlim)) : (!EM || idx < lim));
      T x0 = ok ? v : T(0);
#pragma unroll
      for (int k = 1; k < NT; ++k) {
        idx = i + OFF + k;
        v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
        ok = idx < 0 ? okl : (idx >= P ? (okr && (!EM || idx - P < rlim)) : (!EM || idx < lim));
        x0 = ok ? x0 + v : x0;
      }
      yi = fop(SUB, st.c[0], x0, yi);
    } else {
      const int idx = i + OFF;
      const T v = idx < 0 ? xl[HL + idx] : (idx >= P ? xr[idx - P] : x[idx]);
      const bool ok = idx < 0 ? okl : (idx >= P ? (okr && (!EM || idx - P < rlim)) : (!EM || idx < lim));
      const T f = SUB ? yi - v : yi + v;
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

// Generic kernels: the update of one step, dispatched on its shape index
// (shapes reaching past P pairs are not compiled at this level; the host
// never runs those levels).
template <typename T, int OP, int P, int PA, int I, bool EM = false>
__device__ __forceinline__ void wgen_update(int shape, T (&s)[PA], T (&d)[PA],
                                            const DevStep<T>& st, bool okl, bool okr,
                                            int lim = P, int rlim = P) {
  if constexpr (I < GenTable<OP>::v.n) {
    if (shape == I) {
      constexpr CStep cs = GenTable<OP>::v.s[I];
      if constexpr (cs.left <= P && cs.right <= P) {
        if constexpr (cs.y_is_d)
          wupdate<T, P, PA, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, EM>(
              d, s, st, okl, okr, lim, rlim);
        else
          wupdate<T, P, PA, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, EM>(
              s, d, st, okl, okr, lim, rlim);
      }
      return;
    }
    wgen_update<T, OP, P, PA, I + 1, EM>(shape, s, d, st, okl, okr, lim, rlim);
  }
}

template <typename T, int WI, int OP, int K, int P, int PA, bool EM = false, bool EDGE = false>
__device__ __forceinline__ void wsteps(T (&s)[PA], T (&d)[PA],
                                       const DevProgram<T>& prog, bool okl, bool okr,
                                       int lim = P, int rlim = P,
                                       const WEdge<T>* ed = nullptr) {
  if constexpr (WI == WI_GEN) {
    if constexpr (K == 0) {
      for (int k = 0; k < prog.nsteps; ++k) {
        const DevStep<T>& st = prog.st[k];
        if (st.kind == K_SCALE) {
          const T sm = st.sm, dm = st.dm;
#pragma unroll
          for (int i = 0; i < P; ++i) {
            s[i] = s[i] * sm;
            d[i] = d[i] * dm;
          }
        } else {
          wgen_update<T, OP, P, PA, 0, EM>(st.shape, s, d, st, okl, okr, lim, rlim);
        }
      }
    }
  } else if constexpr (K < cat_nsteps(WI)) {
    constexpr CStep cs = cstep(WI, OP, K);
    const DevStep<T>& st = prog.st[K];
    if constexpr (cs.kind == K_SCALE) {
      const T sm = st.sm, dm = st.dm;
#pragma unroll
      for (int i = 0; i < P; ++i) {
        s[i] = s[i] * sm;
        d[i] = d[i] * dm;
      }
    } else if constexpr (cs.y_is_d) {
      wupdate<T, P, PA, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, EM, EDGE>(
          d, s, st, okl, okr, lim, rlim, ed);
    } else {
      wupdate<T, P, PA, cs.kind, cs.off, cs.ntaps, cs.sub, cs.left, cs.right, EM, EDGE>(
          s, d, st, okl, okr, lim, rlim, ed);
    }
    wsteps<T, WI, OP, K + 1, P, PA, EM, EDGE>(s, d, prog, okl, okr, lim, rlim, ed);
  }
}

// Coarse levels past the register levels (the pairs per lane would drop
// below the steps' reach): the band is compacted onto fewer lanes through
// the row buffer, PC pairs per active lane, and every further level halves
// the active lanes.  Bands this small all use the unswizzled unit layout
// (run length 1), which is what the banded drain and fill use for them.
constexpr int pow2_at_least(int r) {
  int p = 1;
  while (p < r) p <<= 1;
  return p;
}
template <int WI, int OP>
constexpr int compact_pairs() {
  if constexpr (WI == WI_GEN) {
    return 16;  // covers every catalogue reach
  } else {
    return pow2_at_least(cat_reach(WI, OP) > 1 ? cat_reach(WI, OP) : 1);
  }
}

// Active lanes take 2*PC consecutive elements (written with run length
// CHUNK) as PC pairs; the others hold zeros.
template <typename T, int CHUNK, int PC>
__device__ __forceinline__ void take_pairs(T* buf, int lane, int act, T (&cs)[PC], T (&cd)[PC]) {
  T w[2 * PC];
  if (lane < act) {
    read_run<T, CHUNK, 2 * PC>(buf, 2 * PC * lane, w);
  } else {
#pragma unroll
    for (int i = 0; i < 2 * PC; ++i) w[i] = T(0);
  }
#pragma unroll
  for (int i = 0; i < PC; ++i) {
    cs[i] = w[2 * i];
    cd[i] = w[2 * i + 1];
  }
}

// Forward levels lv0 .. levels-1 on a band whose approximation a_lv0 is
// in s, P elements per lane (32 * P elements).
template <typename T, int WI, int OP, int P, int PA, bool EDGE = false>
__device__ __forceinline__ void wcompact_fwd(const T (&s)[PA], T* buf, const DevProgram<T>& prog,
                                             int levels, int lv0, int lane, int bc = BC_ZERO) {
  constexpr int PC = compact_pairs<WI, OP>();
  static_assert(16 * P >= PC, "band too short to compact");
  write_run<T, P, P>(buf, P * lane, s);
  __syncwarp();
  int act = 16 * P / PC;
  T cs[PC], cd[PC];
  take_pairs<T, P, PC>(buf, lane, act, cs, cd);
  __syncwarp();
  for (int lv = lv0; lv < levels; ++lv) {
    const int nb = act * PC;  // pairs of this level's band
    const WEdge<T> ed{&prog, bc, nb};
    wsteps<T, WI, OP, 0, PC, PC, false, EDGE>(cs, cd, prog, lane > 0, lane < act - 1, PC, PC,
                                              &ed);
    if (lane < act) write_run<T, 1, PC>(buf, nb + PC * lane, cd);
    if (lane < act) write_run<T, 1, PC>(buf, PC * lane, cs);
    if (lv + 1 == levels) return;
    __syncwarp();
    act >>= 1;
    take_pairs<T, 1, PC>(buf, lane, act, cs, cd);
    __syncwarp();
  }
}

// Reverse levels levels-1 .. lv0 (coarsest first); leaves a_lv0 in s, P
// elements per lane, for the register levels below.
template <typename T, int WI, int OP, int P, int PA, bool EDGE = false>
__device__ __forceinline__ void wcompact_rev(T (&s)[PA], T* buf, const DevProgram<T>& prog,
                                             int levels, int lv0, int lane, int bc = BC_ZERO) {
  constexpr int PC = compact_pairs<WI, OP>();
  static_assert(16 * P >= PC, "band too short to compact");
  int act = ((16 * P) >> (levels - 1 - lv0)) / PC;
  T cs[PC], cd[PC];
  if (lane < act) {
    read_run<T, 1, PC>(buf, PC * lane, cs);  // a_L
  } else {
#pragma unroll
    for (int i = 0; i < PC; ++i) cs[i] = T(0);
  }
  for (int lv = levels - 1; lv >= lv0; --lv) {
    const int nb = act * PC;
    if (lane < act) {
      read_run<T, 1, PC>(buf, nb + PC * lane, cd);
    } else {
#pragma unroll
      for (int i = 0; i < PC; ++i) cd[i] = T(0);
    }
    const WEdge<T> ed{&prog, bc, nb};
    wsteps<T, WI, OP, 0, PC, PC, false, EDGE>(cs, cd, prog, lane > 0, lane < act - 1, PC, PC,
                                              &ed);
    __syncwarp();  // the band is read before a_lv overwrites it
    if (lane < act) {
      T w[2 * PC];
#pragma unroll
      for (int i = 0; i < PC; ++i) {
        w[2 * i] = cs[i];
        w[2 * i + 1] = cd[i];
      }
      write_run<T, 1, 2 * PC>(buf, 2 * PC * lane, w);
    }
    __syncwarp();
    if (lv > lv0) {
      act <<= 1;
      if (lane < act) {
        read_run<T, 1, PC>(buf, PC * lane, cs);
      } else {
#pragma unroll
        for (int i = 0; i < PC; ++i) cs[i] = T(0);
      }
    }
  }
  read_run<T, 1, P>(buf, P * lane, s);
  __syncwarp();
}

// Forward-stepping levels: band of level LV+1 has 32*P pairs.
template <typename T, int WI, int OP, int P0, int LV, bool EDGE = false>
__device__ __forceinline__ void wfwd(T (&s)[P0], T (&d)[P0], T* buf,
                                     const DevProgram<T>& prog, int levels,
                                     int lane, int lc, int bc = BC_ZERO) {
  constexpr int P = P0 >> LV;
  if constexpr (P >= 1 && P >= kreach(WI, OP)) {
    if (LV < levels) {
      constexpr int NB = 32 * P;  // band length at this level
      const WEdge<T> ed{&prog, bc, NB};
      wsteps<T, WI, OP, 0, P, P0, false, EDGE>(s, d, prog, lane > 0, lane < 31, P, P, &ed);
      write_run<T, P, P>(buf, NB + P * lane, d);
      if (LV + 1 == levels) {
        write_run<T, P, P>(buf, P * lane, s);
        return;
      }
      if constexpr (WI == WI_GEN) {
        // the wavelet's register levels end at lc (run time)
        if (LV + 1 >= lc) {
          wcompact_fwd<T, WI, OP, P, P0, EDGE>(s, buf, prog, levels, LV + 1, lane, bc);
          return;
        }
#pragma unroll
        for (int i = 0; i < P / 2; ++i) {
          d[i] = s[2 * i + 1];
          s[i] = s[2 * i];
        }
        wfwd<T, WI, OP, P0, LV + 1, EDGE>(s, d, buf, prog, levels, lane, lc, bc);
      } else if constexpr (LV + 1 >= reg_max_levels(WI, OP, P0)) {
        wcompact_fwd<T, WI, OP, P, P0, EDGE>(s, buf, prog, levels, LV + 1, lane, bc);
      } else {
#pragma unroll
        for (int i = 0; i < P / 2; ++i) {
          d[i] = s[2 * i + 1];
          s[i] = s[2 * i];
        }
        wfwd<T, WI, OP, P0, LV + 1, EDGE>(s, d, buf, prog, levels, lane, lc, bc);
      }
    }
  }
}

// Reverse-stepping levels, coarsest first (LV counts down).
template <typename T, int WI, int OP, int P0, int LV, bool EDGE = false>
__device__ __forceinline__ void wrev(T (&s)[P0], T (&d)[P0], T* buf,
                                     const DevProgram<T>& prog, int levels,
                                     int lane, int lc, int bc = BC_ZERO) {
  constexpr int P = P0 >> LV;
  if constexpr (LV >= 0) {
    if constexpr (P >= 1 && P >= kreach(WI, OP)) {
      // generic: levels at and past lc ran on compacted lanes
      if (LV < levels && (WI != WI_GEN || LV < lc)) {
        constexpr int NB = 32 * P;
        if (LV + 1 == levels) read_run<T, P, P>(buf, P * lane, s);
        read_run<T, P, P>(buf, NB + P * lane, d);
        const WEdge<T> ed{&prog, bc, NB};
        wsteps<T, WI, OP, 0, P, P0, false, EDGE>(s, d, prog, lane > 0, lane < 31, P, P, &ed);
        if constexpr (LV > 0) {
#pragma unroll
          for (int i = P - 1; i >= 0; --i) {
            s[2 * i + 1] = d[i];
            s[2 * i] = s[i];
          }
        }
      }
    }
    if constexpr (LV > 0) wrev<T, WI, OP, P0, LV - 1, EDGE>(s, d, buf, prog, levels, lane, lc, bc);
  }
}

// Generic instantiation: the compacted reverse levels above register
// level lc (run time), dispatched to the instantiation for its pair count.
template <typename T, int WI, int OP, int P0, int L>
__device__ __forceinline__ void gen_compact_rev(int lc, T (&s)[P0], T* buf,
                                                const DevProgram<T>& prog, int levels,
                                                int lane) {
  if constexpr ((P0 >> L) >= 1) {
    if (lc - 1 == L) {
      wcompact_rev<T, WI, OP, (P0 >> L), P0>(s, buf, prog, levels, lc, lane);
      return;
    }
    gen_compact_rev<T, WI, OP, P0, L + 1>(lc, s, buf, prog, levels, lane);
  }
}

}  // namespace wrow

// Largest number of levels one warp can run on a row of 64*P0 elements.
constexpr int wrow_max_levels(int wi, int op, int p0) {
  const int lc = reg_max_levels(wi, op, p0);
  if (lc < 1) return 0;
  const int reach = cat_reach(wi, op) > 1 ? cat_reach(wi, op) : 1;
  int pc = 1;
  while (pc < reach) pc <<= 1;
  int act = 16 * (p0 >> (lc - 1)) / pc;  // lanes of the first compacted level
  int lv = lc;
  while (act >= 1 && lv < MAX_LEVELS) {
    ++lv;
    act >>= 1;
  }
  return lv;
}

// EDGE: the instantiation for the Constant, Symmetric and Reflect
// boundaries (exact band edges, lw_edge.cuh; compiled wavelets).
template <typename T, int WI, int OP, int P0, bool EDGE = false>
__global__ void __launch_bounds__(128)
    wrow_kernel(const __grid_constant__ WRowParams<T> p) {
  constexpr int N = 64 * P0;                  // row length
  constexpr int EPU = 16 / (int)sizeof(T);    // elements per 16-byte unit
  constexpr int UNITS = N / EPU;
  constexpr bool FWD = (OP == TF_F || OP == TF_IA);
  extern __shared__ __align__(16) unsigned char lw_wrow_smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (row >= p.g.nlines) return;  // whole warps only: no block barriers used
  pdl_wait();  // the previous kernel's results (no global access before)
  pdl_trigger();
  T* buf = reinterpret_cast<T*>(lw_wrow_smem) + (int64_t)warp * N;
  int64_t bin, bout;
  line_base(p.g, row, bin, bout);
  const T* src = p.in + bin;
  T* dst = p.out + bout;

  // Approximation band length after the last level (banded layout).
  const int nbl = N >> p.levels;
  constexpr int SHA = wrow::swz_shift_bytes(2 * P0 * (int)sizeof(T));

  // coalesced fill: chunk layout (forward reads whole runs of 2*P0) or
  // banded layout (reverse reads each level's bands)
#pragma unroll 4
  for (int u = lane; u < UNITS; u += 32) {
    const int sh = FWD ? SHA : wrow::banded_shift<T>(u, nbl);
    const unsigned saddr =
        (unsigned)__cvta_generic_to_shared(buf + wrow::swz(u, sh) * EPU);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr),
                 "l"(src + (int64_t)u * EPU)
                 : "memory");
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncwarp();

  T s[P0], d[P0];
  if constexpr (FWD) {
    T x[2 * P0];
    wrow::read_run<T, 2 * P0, 2 * P0>(buf, 2 * P0 * lane, x);
#pragma unroll
    for (int i = 0; i < P0; ++i) {
      s[i] = x[2 * i];
      d[i] = x[2 * i + 1];
    }
    __syncwarp();
    wrow::wfwd<T, WI, OP, P0, 0, EDGE>(s, d, buf, p.prog, p.levels, lane, p.reg_levels, p.bc);
  } else {
    constexpr int TOP = reg_max_levels(WI, OP, P0) - 1;
    if constexpr (WI != WI_GEN) {
      if (p.levels > TOP + 1)
        wrow::wcompact_rev<T, WI, OP, (P0 >> TOP), P0, EDGE>(s, buf, p.prog, p.levels, TOP + 1,
                                                             lane, p.bc);
    } else {
      if (p.levels > p.reg_levels && p.reg_levels >= 1)
        wrow::gen_compact_rev<T, WI, OP, P0, 0>(p.reg_levels, s, buf, p.prog, p.levels, lane);
    }
    wrow::wrev<T, WI, OP, P0, TOP, EDGE>(s, d, buf, p.prog, p.levels, lane, p.reg_levels, p.bc);
    __syncwarp();
    T x[2 * P0];
#pragma unroll
    for (int i = 0; i < P0; ++i) {
      x[2 * i] = s[i];
      x[2 * i + 1] = d[i];
    }
    wrow::write_run<T, 2 * P0, 2 * P0>(buf, 2 * P0 * lane, x);
  }
  __syncwarp();
  // coalesced drain: banded layout (forward) or chunk layout (reverse)
#pragma unroll 4
  for (int u = lane; u < UNITS; u += 32) {
    const int sh = FWD ? wrow::banded_shift<T>(u, nbl) : SHA;
    const T* q = buf + wrow::swz(u, sh) * EPU;
    if constexpr (sizeof(T) == 4) {
      *reinterpret_cast<float4*>(dst + (int64_t)u * EPU) = *reinterpret_cast<const float4*>(q);
    } else {
      *reinterpret_cast<double2*>(dst + (int64_t)u * EPU) = *reinterpret_cast<const double2*>(q);
    }
  }
}

}  // namespace lw
