// Instantiations and planning of the register-blocked kernel
// (lw_reg_kernel.cuh).  plan_reg_pass() decides whether one axis pass can run
// on the register path and launches it; otherwise the caller uses the
// general line kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda.h>

#include "lw_col.hpp"
#include "lw_col_kernel.cuh"
#include "lw_edge.cuh"
#include "lw_launch.hpp"
#include "lw_reg.hpp"
#include "lw_reg_inst.hpp"
#include "lw_wtile_kernel.cuh"
#include "lw_reg_kernel.cuh"
#include "lw_wrow.hpp"
#include "lw_wrow_kernel.cuh"

namespace lw {

namespace {

// Catalogue indices of the wavelets compiled into the register path.
constexpr int WI_DB2 = 2;     // Daubechies2
constexpr int WI_DB4 = 4;     // Daubechies4
constexpr int WI_CDF97 = 33;  // CDF9_7

template <typename T>
constexpr int p0_of() {
  return sizeof(T) == 4 ? 16 : 8;
}

template <typename T>
RegFn<T> pick(int wi, int op, bool strided, bool tile, int v, bool edge) {
  if constexpr (sizeof(T) == 4)
    return pick_reg_f32(wi, op, strided, tile, v, edge);
  else
    return pick_reg_f64(wi, op, strided, tile, v, edge);
}

bool compiled_wavelet(int wi) {
  return wi == WI_DB2 || wi == WI_DB4 || wi == WI_CDF97;
}

// Shape indices of a catalogue program's steps in the generic kernels'
// table for transform `op`; false if a step has no compiled shape.
template <typename T>
bool set_gen_shapes(DevProgram<T>* p, int op) {
  const GenShapes* g = op == 0 ? &GenTable<0>::v
                     : op == 1 ? &GenTable<1>::v
                     : op == 2 ? &GenTable<2>::v
                               : &GenTable<3>::v;
  for (int k = 0; k < p->nsteps; ++k) {
    DevStep<T>& st = p->st[k];
    st.shape = -1;
    if (st.kind == K_SCALE) continue;
    const CStep c{st.kind, st.y_is_d, st.off, st.ntaps, st.sub, 0, 0};
    for (int i = 0; i < g->n; ++i)
      if (same_shape(g->s[i], c)) {
        st.shape = i;
        break;
      }
    if (st.shape < 0) return false;
  }
  return true;
}

// Whether, at some level, a step's front and back edge ranges overlap (a
// band shorter than the taps reaching into it from both sides): there the
// reference updates the overlapping indices twice (front, then back), which
// the register kernels, which skip out-of-band taps once, do not reproduce.
// Bands of n >> (l + 1) pairs (every level's band a whole number of pairs).
template <typename T>
bool edges_overlap(const DevProgram<T>& prog, int64_t n, int levels) {
  int64_t m = n;  // the level's input band: s of ceil(m / 2), d of floor(m / 2)
  for (int l = 0; l < levels; ++l) {
    const int64_t nd = m / 2, ns = m - nd;
    for (int k = 0; k < prog.nsteps; ++k) {
      const DevStep<T>& st = prog.st[k];
      if (st.kind == K_SCALE) continue;
      const int64_t ny = st.y_is_d ? nd : ns;
      const int64_t n1 = st.nf < ny ? (int64_t)st.nf : ny;
      const int64_t n2 = nd > st.nb ? nd - st.nb : 0;
      if (n1 > n2) return true;
    }
    m = ns;
  }
  return false;
}

// Length of the approximation band after k levels: ceil(n / 2^k).
inline int64_t band_after(int64_t n, int k) { return (n + ((int64_t)1 << k) - 1) >> k; }

// How far from a band end (pairs) the exact edge work of the register
// kernels reaches under boundary bc (lw_edge.cuh): the largest distance from
// the nearer end of any element a step's edge loops read or write, on a band
// long enough that the two ends stay apart.  1 for the Zero boundary (no edge
// work); -1 when the register kernels do not serve bc (Periodic maps to the
// far end) or the reach exceeds their edge window.  A launch runs a level in
// registers only when its chunks hold at least this many pairs.
template <typename T>
int edge_footprint(const DevProgram<T>& prog, int bc) {
  if (bc == BC_ZERO) return 1;
  if (bc != BC_CONSTANT && bc != BC_SYMMETRIC && bc != BC_REFLECT) return -1;
  const int64_t nb = (int64_t)1 << 20;
  int64_t F = 1;
  auto touch = [&](int64_t idx) {
    if (idx < 0 || idx >= nb) return;
    F = std::max<int64_t>(F, idx < nb / 2 ? idx + 1 : nb - idx);
  };
  auto taps_at = [&](const DevStep<T>& st, int64_t j, bool mapped) {
    const int nt = st.kind == K_UNIT ? 1 : st.ntaps;
    for (int t = 0; t < nt; ++t)
      touch(mapped ? host_bc_index(bc, j + t, nb) : j + t);
  };
  for (int k = 0; k < prog.nsteps; ++k) {
    const DevStep<T>& st = prog.st[k];
    if (st.kind == K_SCALE) continue;
    const int64_t n1 = std::min<int64_t>(st.nf, nb);
    const int64_t n2 = nb > st.nb ? nb - st.nb : 0;
    if (prog.normal) {
      for (int64_t i = 0; i < n1; ++i) {
        touch(i);
        taps_at(st, i + st.off, true);
      }
      for (int64_t i = n2; i < nb; ++i) {
        touch(i);
        taps_at(st, i + st.off, true);
      }
      continue;
    }
    if (st.kind == K_UNIT) {
      for (int64_t i = st.fold_off, j = 0; i < 0 && j < nb; ++i, ++j) {
        const int64_t io = host_bc_index(bc, i, nb);
        if (io < nb && io != i) {
          touch(io);
          touch(j);
        }
      }
    } else {
      for (int64_t i = st.fold_off, j = 1 - st.ntaps; i < 0; ++i, ++j) {
        const int64_t io = host_bc_index(bc, i, nb);
        if (io < nb && io != i) {
          touch(io);
          taps_at(st, j, false);
        }
      }
    }
    for (int64_t i = nb, j = nb + st.off; i < nb - st.off; ++i, ++j) {
      const int64_t io = host_bc_index(bc, i, nb);
      if (io < nb && io != i) {
        touch(io);
        taps_at(st, j, false);
      }
    }
  }
  return F > edge::kEdge ? -1 : (int)F;
}

// Register levels a launch with p0 pairs per chunk at its first level may
// run under edge footprint F (every level's chunks at least F pairs).
int edge_levels(int p0, int F) {
  int l = 0;
  for (int p = p0; p >= F && p >= 1; p >>= 1) ++l;
  return l;
}

// The host-resolved program must have exactly the compile-time structure.
template <typename T>
bool structure_matches(const DevProgram<T>& prog, int wi, int op) {
  if (prog.nsteps != cat_nsteps(wi)) return false;
  for (int k = 0; k < prog.nsteps; ++k) {
    const CStep c = cstep(wi, op, k);
    const DevStep<T>& s = prog.st[k];
    if (s.kind != c.kind || s.ntaps != c.ntaps) return false;
    if (c.kind == K_SCALE) continue;
    if (s.y_is_d != c.y_is_d || s.off != c.off || s.sub != c.sub) return false;
  }
  return true;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

int sm_count() {
  static int n[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return 148;
  }
  if (!n[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    n[dev] = v;
  }
  return n[dev];
}

// Unit-stride rows whose line bases are all 16-byte aligned.
template <typename T>
bool rows_vectorisable(const LineGeom& g, const T* in, const T* out) {
  if (g.sin != 1 || g.sout != 1) return false;
  if (!aligned16(in) || !aligned16(out)) return false;
  for (int d = 0; d < g.nother; ++d)
    if (((g.oin[d] * (int64_t)sizeof(T)) & 15) || ((g.oout[d] * (int64_t)sizeof(T)) & 15))
      return false;
  return true;
}

// Two adjacent lines per lane (float only): even line count, even strides
// and 8-byte aligned bases so every lane access is one aligned float2.
template <typename T>
int lane_width(const LineGeom& g, const T* in, const T* out) {
  if (sizeof(T) != 4) return 1;
  if (g.nlines % 2 || g.nother < 1 || (g.oshape[0] % 2)) return 1;
  if ((g.sin % 2) || (g.sout % 2)) return 1;
  for (int d = 1; d < g.nother; ++d)
    if ((g.oin[d] % 2) || (g.oout[d] % 2)) return 1;
  if ((reinterpret_cast<uintptr_t>(in) & 7) || (reinterpret_cast<uintptr_t>(out) & 7))
    return 1;
  return 2;
}

// Lines adjacent in memory along the fastest other dim (both sides).
bool lines_adjacent(const LineGeom& g) {
  return g.nother >= 1 && g.oin[0] == 1 && g.oout[0] == 1;
}

template <typename T>
size_t reg_smem(int hmax, int block, int lines_cta, int64_t m_coarse,
                bool coarse, int v = 1) {
  size_t b = (size_t)4 * hmax * block * sizeof(T) * v + 16;
  if (coarse)  // A and B, each m elements per line (coarse_forward/_reverse)
    b += (size_t)lines_cta * (size_t)(2 * m_coarse) * sizeof(T);
  return b;
}

template <typename T>
int launch_whole(const RegPassArgs<T>& a, const LineGeom& g, const T* in,
                 T* out, int levels, bool strided, cudaStream_t stream,
                 RegStats* stats) {
  constexpr int P0 = p0_of<T>();
  const int wi = a.wi, op = a.op;
  const int64_t n = g.n;
  if (n % (2 * P0)) return 0;
  const int64_t tpl = n / (2 * P0);
  const int F = edge_footprint(*a.prog, a.bc);
  if (F < 0) return 0;
  const int maxreg = std::min(reg_max_levels(wi, op, P0), edge_levels(P0, F));
  const int nreg = levels < maxreg ? levels : maxreg;
  if (nreg < 1) return 0;
  int lpc = 1, block;
  int v = 1;
  if (strided) {
    if (tpl > 16) return 0;
    v = lane_width<T>(g, in, out);
    lpc = 32;
    // short bands of few lines: narrower line groups keep every SM busy
    const int64_t want = (int64_t)sm_count();
    if ((g.nlines + 63) / 64 < want) v = 1;
    while (lpc > 8 && (g.nlines + lpc * v - 1) / (lpc * v) < want) lpc /= 2;
    block = lpc * (int)tpl;
  } else {
    if (tpl > 512) return 0;
    lpc = (int)(256 / tpl);
    if (lpc < 1) lpc = 1;
    if (lpc > g.nlines) lpc = (int)g.nlines;
    block = lpc * (int)tpl;
  }
  const int lines_cta = lpc * v;
  const int64_t m = n >> nreg;
  const bool coarse = nreg < levels;
  const int hmax = cat_reach(wi, op) > 0 ? cat_reach(wi, op) : 1;
  const size_t smem = reg_smem<T>(hmax, block, lines_cta, m, coarse, v);
  if (smem > kMaxDynSmem) return 0;
  RegParams<T> p;
  std::memset(&p, 0, sizeof(p));
  p.l2hint = l2_hint_code();
  p.bc = a.bc;
  p.in = in;
  p.out = out;
  p.g = g;
  p.levels = levels;
  p.nreg = nreg;
  p.tpl = (int)tpl;
  p.lpc = lpc;
  p.vec = (!strided && rows_vectorisable(g, in, out)) ? 1 : 0;
  p.coarse_pitch = (int)m;
  p.coarse_pitch_b = (int)m;
  p.prog = *a.prog;
  const int64_t groups = (g.nlines + lines_cta - 1) / lines_cta;
  if (groups > 0x7fffffffLL) return 0;
  RegFn<T> fn = pick<T>(wi, op, strided, false, v, a.bc != BC_ZERO || edge_kernels_always());
  if (!fn) return 0;
  cudaError_t e = fn(p, (int)groups, block, smem, stream);
  if (e != cudaSuccess) return -(int)e - 1000;
  counted(stats, KF_REG);
  return 1;
}

// Contiguous rows of 64 * P0 elements, every level in one warp's registers
// (or, for float32 rows of 2048 and 4096, in a pair of warps' registers).
template <typename T>
int launch_wrow(const RegPassArgs<T>& a, cudaStream_t stream, RegStats* stats) {
  const LineGeom& g = a.g;
  if (!rows_vectorisable(g, a.in, a.out)) return 0;
  // catalogue wavelets without a compiled kernel: the generic instantiation,
  // every register level the wavelet's reach allows (no compacted levels)
  const bool gen = !compiled_wavelet(a.wi);
  // Constant / Symmetric / Reflect: the one-warp kernel's exact-edge
  // instantiation, compiled wavelets only
  const bool zero = a.bc == BC_ZERO;
  if (!zero && gen) return 0;
  const int F = edge_footprint(*a.prog, a.bc);
  if (F < 0) return 0;
  if constexpr (sizeof(T) == 4) {
    const int64_t q0 = g.n / 128;
    // non-Zero boundaries: every level's lanes hold the edge reach
    const bool edge_fits = zero || (a.levels >= 1 && (q0 >> (a.levels - 1)) >= F);
    if (!gen && edge_fits && wrow2_enabled() && g.n % 128 == 0 && (q0 == 16 || q0 == 32) &&
        wrow2_levels_f32(a.wi, a.op, (int)q0) >= a.levels) {
      WRowParams<T> p;
      std::memset(&p, 0, sizeof(p));
      p.in = a.in;
      p.out = a.out;
      p.g = g;
      p.levels = a.levels;
      p.l2hint = l2_hint_code();
      p.bc = a.bc;
      p.prog = *a.prog;
      const size_t smem = (size_t)4 * (size_t)g.n * sizeof(T);
      const int64_t grid = std::min<int64_t>((g.nlines + 1) / 2,
                                             (int64_t)sm_count() * wrow2_resident_ctas((int)q0));
      if (grid <= 0x7fffffffLL) {
        cudaError_t e = launch_wrow2_f32(a.wi, a.op, (int)q0, p, (int)grid, smem, stream,
                                         !zero || edge_kernels_always());
        if (e != cudaSuccess) return -(int)e - 1000;
        counted(stats, KF_WROW2);
        return 1;
      }
    }
  }
  if (g.n % 64) return 0;
  const int64_t p0 = g.n / 64;
  const int maxp0 = sizeof(T) == 4 ? 64 : 32;
  if (p0 < 8 || p0 > maxp0 || (p0 & (p0 - 1))) return 0;
  // generic: the wavelet's register levels, then compacted lanes of 16
  // pairs each, halving per level down to one lane
  const int lc = gen ? reg_max_levels(a.wi, a.op, (int)p0) : 0;
  int lv;
  if (gen) {
    lv = lc;
    if (lc >= 1)
      for (int64_t act = (int64_t)p0 >> (lc - 1); act >= 1; act >>= 1) ++lv;
  } else {
    lv = sizeof(T) == 4 ? wrow_levels_f32(a.wi, a.op, (int)p0) : wrow_levels_f64(a.wi, a.op, (int)p0);
  }
  if (lc < 0 || lv < a.levels || (gen && lc < 1)) return 0;
  if (!zero) {
    // every level's lanes must hold the edge work's reach: the register
    // levels' pairs, then the compacted lanes' pairs
    const int lreg = reg_max_levels(a.wi, a.op, (int)p0);
    for (int j = 0; j < std::min(lreg, a.levels); ++j)
      if (((int)p0 >> j) < F) return 0;
    if (a.levels > lreg) {
      const int reach = std::max(cat_reach(a.wi, a.op), 1);
      int pc = 1;
      while (pc < reach) pc <<= 1;
      if (pc < F) return 0;
    }
  }
  WRowParams<T> p;
  std::memset(&p, 0, sizeof(p));
  p.in = a.in;
  p.out = a.out;
  p.g = g;
  p.levels = a.levels;
  p.bc = a.bc;
  p.prog = *a.prog;
  if (gen && !set_gen_shapes(&p.prog, a.op)) return 0;
  p.reg_levels = lc;
  const int wk = gen ? WI_GEN : a.wi;
  const int warps = 4;
  const size_t smem = (size_t)warps * (size_t)g.n * sizeof(T);
  if (smem > kMaxDynSmem) return 0;
  const int64_t grid = (g.nlines + warps - 1) / warps;
  if (grid > 0x7fffffffLL) return 0;
  cudaError_t e;
  if constexpr (sizeof(T) == 4)
    e = launch_wrow_f32(wk, a.op, (int)p0, p, (int)grid, 32 * warps, smem, stream,
                        (!zero || edge_kernels_always()) && !gen);
  else
    e = launch_wrow_f64(wk, a.op, (int)p0, p, (int)grid, 32 * warps, smem, stream,
                        (!zero || edge_kernels_always()) && !gen);
  if (e != cudaSuccess) return -(int)e - 1000;
  counted(stats, KF_WROW);
  return 1;
}

// Contiguous rows longer than one warp holds: every level on windows of
// 64 * P0 samples with halos (lw_wtile_kernel.cuh), one launch.
template <typename T>
int launch_wtile(const RegPassArgs<T>& a, cudaStream_t stream, RegStats* stats) {
  const LineGeom& g = a.g;
  if (!wtile_enabled() || a.in_place) return 0;  // windows read other windows' input
  if (!rows_vectorisable(g, a.in, a.out)) return 0;
  const int p0 = wtile_pairs((int)sizeof(T));
  const int64_t W = 64 * (int64_t)p0;
  const int64_t n = g.n;
  if (a.levels < 1 || a.levels > wtile_levels(a.wi, a.op, (int)sizeof(T))) return 0;
  // every level's band a whole number of pairs: n a multiple of 2^levels;
  // lengths that are not multiples of a lane's pairs mask the band's end
  // (rows up to one window are one window)
  if (n < 2 || n % ((int64_t)1 << a.levels)) return 0;
  const bool end_mask = (n % (2 * p0)) != 0;
  if (!end_mask && n <= W) return 0;  // the warp-per-row kernel takes these
  // halo: the samples k levels corrupt from a window edge, whole lanes
  int64_t need = 0;
  const int lh = cat_level_halo(a.wi, a.op);
  for (int l = 1; l <= a.levels; ++l) need += (int64_t)lh << l;
  const int64_t halo = (need + 2 * p0 - 1) / (2 * p0) * (2 * p0);
  const int64_t tile = W - 2 * halo;
  if (tile < W / 4) return 0;
  WTileParams<T> p;
  std::memset(&p, 0, sizeof(p));
  p.in = a.in;
  p.out = a.out;
  p.g = g;
  p.tile = tile;
  p.halo = halo;
  p.ntiles = (n + tile - 1) / tile;
  p.levels = a.levels;
  p.prog = *a.prog;
  const bool gen = !compiled_wavelet(a.wi);
  if (gen && !set_gen_shapes(&p.prog, a.op)) return 0;
  const int wk = gen ? WI_GEN : a.wi;
  const int warps = 4;
  const int64_t grid = (g.nlines * p.ntiles + warps - 1) / warps;
  if (grid > 0x7fffffffLL) return 0;
  const size_t smem = (size_t)warps * (size_t)W * sizeof(T);
  cudaError_t e;
  if constexpr (sizeof(T) == 4) e = launch_wtile_f32(wk, a.op, end_mask, p, (int)grid, smem, stream);
  else e = launch_wtile_f64(wk, a.op, end_mask, p, (int)grid, smem, stream);
  if (e != cudaSuccess) return -(int)e - 1000;
  counted(stats, KF_WTILE);
  return 1;
}

// Long lines: tile launch of the first k levels, then a whole-line launch of
// the rest on the (short) approximation band held in `tmp`.
template <typename T>
int launch_tiled(const RegPassArgs<T>& a, cudaStream_t stream,
                 RegStats* stats) {
  constexpr int P0 = p0_of<T>();
  const LineGeom& g = a.g;
  const int wi = a.wi, op = a.op;
  const int64_t n = g.n;
  if (a.in_place) return 0;  // tiles would overwrite other tiles' input
  if (!lines_adjacent(g)) return 0;
  if (n % (2 * P0)) return 0;
  const int F = edge_footprint(*a.prog, a.bc);
  if (F < 0) return 0;
  const int maxreg = std::min(reg_max_levels(wi, op, P0), edge_levels(P0, F));
  // choose k so that the approximation band fits a strided whole-line launch
  int k = 0;
  for (int kk = 1; kk <= maxreg && kk <= a.levels; ++kk) {
    if ((n % ((int64_t)1 << kk)) != 0) break;
    k = kk;
    const int64_t m = n >> kk;
    if (m % (2 * P0) == 0 && m / (2 * P0) <= 16) break;
  }
  if (k < 1) return 0;
  const int64_t m = n >> k;
  // halo: what k levels consume, rounded up to whole chunks
  int64_t need = 0;
  const int lh = cat_level_halo(wi, op);
  for (int l = 1; l <= k; ++l) need += (int64_t)lh << l;
  const int64_t chunk = 2 * P0;
  const int64_t halo = (need + chunk - 1) / chunk * chunk;
  const int64_t hchunks = halo / chunk;
  int64_t ichunks = 16 - 2 * hchunks;  // 512 threads at most
  if (ichunks < 4) return 0;
  if (ichunks * chunk > n) ichunks = n / chunk;
  const int64_t tile = ichunks * chunk;
  const int tpl = (int)(ichunks + 2 * hchunks);
  const int block = 32 * tpl;
  const int hmax = cat_reach(wi, op) > 0 ? cat_reach(wi, op) : 1;
  const int v = lane_width<T>(g, a.in, a.out);
  const size_t smem = reg_smem<T>(hmax, block, 32 * v, 0, false, v);
  const int64_t ntiles = (n + tile - 1) / tile;
  const int64_t groups = (g.nlines + 32 * v - 1) / (32 * v);
  if (groups * ntiles > 0x7fffffffLL) return 0;
  // the whole-line launch on the approximation band must be possible too
  if (a.levels > k && ((m % (2 * P0)) || (m / (2 * P0)) > 16)) return 0;

  T* tmp = nullptr;
  cudaError_t e = cudaSuccess;
  if (a.levels > k) {
    const size_t tbytes = (size_t)g.nlines * (size_t)m * sizeof(T);
    e = scratch_alloc((void**)&tmp, tbytes, stream);
    if (e != cudaSuccess) return -(int)e - 1000;
  }

  RegParams<T> p;
  std::memset(&p, 0, sizeof(p));
  p.l2hint = l2_hint_code();
  p.bc = a.bc;
  p.g = g;
  p.tmp = tmp;
  p.tmp_line = 1;          // tmp is [position][line]: lines adjacent
  p.tmp_pos = g.nlines;
  p.nreg = k;
  p.levels = k;
  p.tpl = tpl;
  p.lpc = 32;
  p.tile = tile;
  p.halo = halo;
  p.ntiles = ntiles;
  p.prog = *a.prog;
  RegFn<T> tfn = pick<T>(wi, op, true, true, v, a.bc != BC_ZERO || edge_kernels_always());
  if (!tfn) {
    if (tmp) scratch_free(tmp, stream);
    return 0;
  }
  // geometry of the approximation band in tmp: one other dim of nlines
  // lines (line index L = linear line index of the pass)
  LineGeom gt;
  std::memset(&gt, 0, sizeof(gt));
  gt.n = m;
  gt.nlines = g.nlines;
  gt.nother = g.nother;
  int64_t acc = 1;
  for (int d = 0; d < g.nother; ++d) {
    gt.oshape[d] = g.oshape[d];
    gt.oin[d] = acc;
    gt.oout[d] = acc;
    acc *= g.oshape[d];
  }
  int rc = 1;
  const bool fwd = (op == TF_F || op == TF_IA);
  const bool more = a.levels > k;  // levels left for the whole-line launch
  p.levels = a.levels;
  p.in = a.in;
  p.out = a.out;
  if (fwd) {
    e = tfn(p, (int)(groups * ntiles), block, smem, stream);
    if (e != cudaSuccess) rc = -(int)e - 1000;
    else counted(stats, KF_REG);
    if (rc == 1 && more) {
      // levels k+1..: tmp -> the first m positions of every output line
      LineGeom g2 = gt;
      g2.sin = g.nlines;
      g2.sout = g.sout;
      for (int d = 0; d < g.nother; ++d) g2.oout[d] = g.oout[d];
      int r2 = launch_whole<T>(a, g2, tmp, a.out, a.levels - k, true, stream, stats);
      if (r2 != 1) rc = r2 == 0 ? -2 : r2;
    }
  } else {
    if (more) {
      // coarse levels first: the first m positions of every input line -> tmp
      LineGeom g2 = gt;
      g2.sin = g.sin;
      g2.sout = g.nlines;
      for (int d = 0; d < g.nother; ++d) g2.oin[d] = g.oin[d];
      int r2 = launch_whole<T>(a, g2, a.in, tmp, a.levels - k, true, stream, stats);
      if (r2 != 1) rc = r2 == 0 ? -2 : r2;
    }
    if (rc == 1) {
      e = tfn(p, (int)(groups * ntiles), block, smem, stream);
      if (e != cudaSuccess) rc = -(int)e - 1000;
      else counted(stats, KF_REG);
    }
  }
  if (tmp) scratch_free(tmp, stream);
  return rc;
}

// Device word the TMA-staged kernel sets when a staging wait gives up.
int32_t* col_error_flag() {
  static int32_t* flag[kMaxDevices] = {};
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!flag[dev]) {
    if (cudaMalloc((void**)&flag[dev], sizeof(int32_t)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    cudaMemset(flag[dev], 0, sizeof(int32_t));
  }
  return flag[dev];
}

// cuTensorMapEncodeTiled from the driver, looked up through the runtime so
// that the library does not link libcuda (it loads on machines without a
// driver; only the GPU paths need one).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000,
                                         cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  }
  return fn;
}

bool encode_rows(CUtensorMap* m, const void* base, int rank, const cuuint64_t* dims,
                 const cuuint64_t* strides, cuuint32_t box_x, cuuint32_t box_y,
                 int elem_bytes, cuuint32_t box_z = 1) {
  EncodeTiledFn enc = encode_tiled_fn();
  if (!enc) return false;
  const cuuint32_t box[3] = {box_x, box_y, box_z};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
             (cuuint32_t)rank, const_cast<void*>(base),
             dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T>
int band_pass(const RegPassArgs<T>& a, const LineGeom& g2, const T* in, T* out, int levels,
              cudaStream_t stream, RegStats* stats);

// Levels of one launch of the TMA-staged kernel on lines of n samples and
// its window geometry: whole lines of up to 512 (k = the register levels,
// fewer when the band must again be a multiple of 32 long), or 512-sample
// windows with halos (the smallest k whose band fits whole lines, else the
// register levels).
template <typename T>
bool col_levels_plan(int wi, int op, int64_t n, int levels, int F, int* k_out, int64_t* tile,
                     int64_t* halo, int64_t* ntr) {
  const int maxreg =
      std::min({reg_max_levels(wi, op, COL_P0), COL_MAXK, edge_levels(COL_P0, F)});
  int k = 0;
  if (n <= COL_ROWS) {
    k = std::min(levels, maxreg);
    // levels past k run on the approximation band: on the whole-line
    // register kernel when its lines fit one (n <= 32 * p0), else here
    // again, which needs band lines a multiple of 32 long (float64 lines
    // of 512 with more levels than the registers hold)
    if (levels > k && n / (2 * p0_of<T>()) > 16)
      while (k > 0 && (band_after(n, k) % 32)) --k;
    *tile = n;
    *halo = 0;
    *ntr = 1;
  } else {
    for (int kk = 1; kk <= maxreg && kk <= levels; ++kk) {
      k = kk;
      const int64_t m = band_after(n, kk);
      if (m % 32 == 0 && m / 32 <= 16) break;
    }
    int64_t need = 0;
    const int lh = cat_level_halo(wi, op);
    for (int l = 1; l <= k; ++l) need += (int64_t)lh << l;
    *halo = (need + 31) / 32 * 32;
    *tile = COL_ROWS - 2 * *halo;
    if (*tile < 128) return false;
    *ntr = (n + *tile - 1) / *tile;
  }
  *k_out = k;
  return k >= 1;
}

// Whether a pass of `levels` levels on lines of n samples runs through to
// the end as a chain of launches of the TMA-staged kernel (each later one on
// the previous one's approximation band; windowed bands chain again), or,
// for compiled wavelets, ends on the whole-line register kernel.  Checked
// before the first launch, so no launch is left without its band pass.
template <typename T>
bool col_chain_ok(int wi, int op, int64_t n, int levels, int F, int depth) {
  // lines a multiple of 32 long, or (the end-masked instantiation: a band
  // ends inside a chunk) of any length under the Zero boundary (F == 1),
  // else of a multiple of 2^levels
  if (depth > 8 || (n % 32 && F != 1 && n % ((int64_t)1 << levels))) return false;
  int k;
  int64_t tile, halo, ntr;
  if (!col_levels_plan<T>(wi, op, n, levels, F, &k, &tile, &halo, &ntr)) return false;
  if (levels == k) return true;
  const int64_t m = band_after(n, k);
  if (col_chain_ok<T>(wi, op, m, levels - k, F, depth + 1)) return true;
  constexpr int P0 = p0_of<T>();
  return compiled_wavelet(wi) && m % (2 * P0) == 0 && m / (2 * P0) <= 16 &&
         edge_levels(P0, F) >= 1;
}

// Strided pass (float32 or float64) on the TMA-staged persistent kernel:
// whole lines of up to 512 samples (several 3D slices per window when they
// are short), or 512-sample windows with halos on longer lines; the levels
// beyond the first k run as further launches on the approximation band
// (band_pass).  Catalogue wavelets without compiled kernels use the generic
// instantiations.  Returns 0 when the pass does not qualify.
template <typename T>
int launch_col(const RegPassArgs<T>& a, cudaStream_t stream, RegStats* stats,
               bool allow_ldg) {
  {
    constexpr int EB = (int)sizeof(T);
    const LineGeom& g = a.g;
    if (!col_enabled()) return 0;
    if (g.sin <= 1) return 0;
    if (!lines_adjacent(g) || g.nother > 2) return 0;
    if (g.nother == 2 && g.oin[1] <= 0) return 0;
    const int64_t ncols = g.oshape[0];
    // TMA wants strides that are multiples of 16 bytes, a 16-byte aligned
    // base, and (a line count that is not a multiple of 32: the last strip
    // is partial) band-buffer boxes starting on 16 bytes at outer * ncols +
    // col0; otherwise the plain-load instantiation stages the tiles (Zero
    // boundary)
    const bool ldg = ((g.sin * EB) & 15) ||
                     (ncols % COL_LANES && (ncols < COL_LANES || ((ncols * EB) & 15))) ||
                     (g.nother == 2 && ((g.oin[1] * EB) & 15)) || !aligned16(a.in);
    if (ldg && (a.bc != BC_ZERO || !allow_ldg)) return 0;
    const int64_t n = g.n;
    // lines whose length is not a multiple of 32: the end-masked
    // instantiation, one line per lane (Zero boundary, any length: bands of
    // odd length at some level have an s band one longer than the d band)
    const bool em = (n % 32) != 0 || ldg;
    // exact band edges of the non-Zero boundaries need whole chunks
    const int F = edge_footprint(*a.prog, a.bc);
    if (F < 0 || (em && a.bc != BC_ZERO)) return 0;
    const int wi = a.wi, op = a.op;
    // two adjacent lines per lane (packed FP32x2) when the line groups and
    // every line base of the output stay 8-byte aligned
    int v = 1;
    if (EB == 4 && col_packed() && ncols % (2 * COL_LANES) == 0 && (g.sout % 2) == 0 &&
        (g.nother < 2 || (g.oout[1] % 2) == 0) && (reinterpret_cast<uintptr_t>(a.out) & 7) == 0)
      v = 2;
    if (n > COL_ROWS && a.in_place) return 0;  // windows would overwrite other windows' input
    int k = 0;
    int64_t tile, halo, ntr;
    if (!col_levels_plan<T>(wi, op, n, a.levels, F, &k, &tile, &halo, &ntr)) return 0;
    const int64_t nouter = g.nother == 2 ? g.oshape[1] : 1;
    // short whole lines of a 3D view: a tile stacks 512/n consecutive outer
    // slices (the staging window stays full)
    int stack = 1;
    // (each slice whole chunks: a chunk never straddles two slices)
    if (col_stacked() && !em && n <= COL_ROWS / 2 && COL_ROWS % n == 0 && g.nother == 2 &&
        nouter >= 2)
      stack = (int)(COL_ROWS / n);
    const int64_t ngroups = (nouter + stack - 1) / stack;
    // packed lanes only while they still give every SM a tile
    if (v == 2 && ncols / (2 * COL_LANES) * ntr * ngroups < sm_count())
      v = 1;
    // catalogue wavelets without compiled kernels: the generic instantiation
    // (reach up to its exchange width), and the band levels must fit one
    // more launch of it
    const bool gen = !compiled_wavelet(wi);
    // reach above the generic exchange width: the wide instantiation
    // (float32, one line per lane)
    const bool wide = gen && cat_reach(wi, op) > kGenHmax;
    if (wide && cat_reach(wi, op) > kGenWideHmax) return 0;
    if (wide) v = 1;
    const int wk = wide ? WI_GENW : (gen ? WI_GEN : wi);
    ColFn<T> fn;
    if (em) v = 1;
    // the exact-edge instantiation packs one line per lane (with two, its
    // edge work overflows the registers)
    const bool edge_inst = (a.bc != BC_ZERO || edge_kernels_always()) && compiled_wavelet(wi) && !em;
    if (edge_inst) v = 1;
    if constexpr (sizeof(T) == 4)
      fn = ldg ? pick_col_ldg_f32(wk, op) : pick_col_f32(wk, op, v, em, edge_inst);
    else
      fn = ldg ? pick_col_ldg_f64(wk, op) : pick_col_f64(wk, op, em, edge_inst);
    if (!fn) return 0;
    const int64_t m = band_after(n, k);
    const bool more = a.levels > k;
    if (more && !col_chain_ok<T>(wi, op, n, a.levels, F, 0)) return 0;
    if (!more && a.levels != k) return 0;
    int32_t* err = col_error_flag();
    if (!err) return 0;

    T* tmp = nullptr;
    if (more) {
      cudaError_t e = scratch_alloc((void**)&tmp, (size_t)g.nlines * m * sizeof(T), stream);
      if (e != cudaSuccess) return -(int)e - 1000;
    }
    ColParams<T> cp;
    std::memset(&cp, 0, sizeof(cp));
    const int rank = g.nother == 2 ? 3 : 2;
    const cuuint64_t dims[3] = {(cuuint64_t)ncols, (cuuint64_t)n,
                                (cuuint64_t)(g.nother == 2 ? g.oshape[1] : 1)};
    const cuuint64_t strides[2] = {(cuuint64_t)g.sin * EB,
                                   (cuuint64_t)(g.nother == 2 ? g.oin[1] : 0) * EB};
    bool ok = true;
    const cuuint32_t bx = (cuuint32_t)(COL_LANES * v);
    const bool fwd_op = (op == TF_F || op == TF_IA);
    if (ldg) {
      // plain-load staging: no tensor maps
    } else if (stack > 1) {
      // forward: two boxes of stack/2 slices x n rows; reverse: region l of
      // every slice (n >> l rows) in one box of all the slices
      if (fwd_op) {
        ok = encode_rows(&cp.tm_rows[0], a.in, rank, dims, strides, bx, (cuuint32_t)n, EB,
                         (cuuint32_t)(stack / 2));
      } else {
        for (int i = 0; i < k && ok; ++i)
          ok = encode_rows(&cp.tm_rows[i], a.in, rank, dims, strides, bx,
                           (cuuint32_t)(n >> (i + 1)), EB, (cuuint32_t)stack);
      }
    } else {
      for (int i = 0; i < k && ok; ++i)
        ok = encode_rows(&cp.tm_rows[i], a.in, rank, dims, strides, bx, (cuuint32_t)(256 >> i),
                         EB);
    }
    if (ldg) {
    } else if (ok && more && stack > 1) {
      // the band buffer [position][line] viewed as {line in slice, position,
      // slice}
      const cuuint64_t tdims[3] = {(cuuint64_t)ncols, (cuuint64_t)m, (cuuint64_t)nouter};
      const cuuint64_t tstr[2] = {(cuuint64_t)g.nlines * EB, (cuuint64_t)ncols * EB};
      ok = encode_rows(&cp.tm_tmp, tmp, 3, tdims, tstr, bx, (cuuint32_t)m, EB,
                       (cuuint32_t)stack);
    } else if (ok && more) {
      const cuuint64_t tdims[2] = {(cuuint64_t)g.nlines, (cuuint64_t)m};
      const cuuint64_t tstr[1] = {(cuuint64_t)g.nlines * EB};
      ok = encode_rows(&cp.tm_tmp, tmp, 2, tdims, tstr, bx, (cuuint32_t)(COL_ROWS >> k), EB);
    }
    if (!ok) {
      if (tmp) scratch_free(tmp, stream);
      return 0;
    }
    RegParams<T>& r = cp.r;
    r.l2hint = l2_hint_code();
    r.bc = a.bc;
    r.in = a.in;
    r.out = a.out;
    r.tmp = tmp;
    r.tmp_line = 1;
    r.tmp_pos = g.nlines;
    r.g = g;
    r.levels = a.levels;
    r.nreg = k;
    r.tpl = COL_CHUNKS;
    r.lpc = COL_LANES;
    r.tile = tile;
    r.halo = halo;
    r.ntiles = ntr;
    r.prog = *a.prog;
    if (gen && !set_gen_shapes(&r.prog, op)) {
      if (tmp) scratch_free(tmp, stream);
      return 0;
    }
    cp.ncols = ncols;
    cp.nouter = nouter;
    cp.ntr = ntr;
    cp.ntiles = (ncols + COL_LANES * v - 1) / (COL_LANES * v) * ntr * ngroups;
    cp.stack = stack;
    cp.rank3 = rank == 3;
    cp.a_from_tmp = more ? 1 : 0;
    cp.spin_limit = 1 << 22;
    cp.row_order = col_row_order() ? 1 : 0;
    cp.err = err;
    const int hmax = wide ? kGenWideHmax
                     : gen ? kGenHmax
                           : (cat_reach(wi, op) > 0 ? cat_reach(wi, op) : 1);
    const size_t smem = col_smem_bytes(hmax, v, EB, (EB == 8 && wide) ? 1 : 2);
    if (smem > kMaxDynSmem) {
      if (tmp) scratch_free(tmp, stream);
      return 0;
    }
    const int grid = (int)std::min<int64_t>(cp.ntiles, sm_count());

    // band geometry: one other dim of nlines lines in tmp [position][line]
    LineGeom gt;
    std::memset(&gt, 0, sizeof(gt));
    gt.n = m;
    gt.nlines = g.nlines;
    gt.nother = g.nother;
    int64_t acc = 1;
    for (int d = 0; d < g.nother; ++d) {
      gt.oshape[d] = g.oshape[d];
      gt.oin[d] = acc;
      gt.oout[d] = acc;
      acc *= g.oshape[d];
    }
    const bool fwd = (op == TF_F || op == TF_IA);
    int rc = 1;
    cudaError_t e = cudaSuccess;
    if (!fwd && more) {
      LineGeom g2 = gt;
      g2.sin = g.sin;
      g2.sout = g.nlines;
      for (int d = 0; d < g.nother; ++d) g2.oin[d] = g.oin[d];
      const int r2 = band_pass<T>(a, g2, a.in, tmp, a.levels - k, stream, stats);
      if (r2 == 0) {
        // nothing launched yet: the caller's fallback takes the whole pass
        scratch_free(tmp, stream);
        return 0;
      }
      if (r2 != 1) rc = r2;
    }
    if (rc == 1) {
      e = fn(cp, grid, smem, stream);
      if (e != cudaSuccess) rc = -(int)e - 1000;
      else counted(stats, KF_COL);
    }
    if (rc == 1 && fwd && more) {
      LineGeom g2 = gt;
      g2.sin = g.nlines;
      g2.sout = g.sout;
      for (int d = 0; d < g.nother; ++d) g2.oout[d] = g.oout[d];
      const int r2 = band_pass<T>(a, g2, tmp, a.out, a.levels - k, stream, stats);
      if (r2 != 1) rc = r2 == 0 ? -2 : r2;
    }
    if (tmp) scratch_free(tmp, stream);
    return rc;
  }
}

// The levels past a tile launch, on the approximation band (lines adjacent
// in memory on at least one side): the TMA-staged kernel when the band
// qualifies (whole lines of up to 512), else the register kernel.
template <typename T>
int band_pass(const RegPassArgs<T>& a, const LineGeom& g2, const T* in, T* out, int levels,
              cudaStream_t stream, RegStats* stats) {
  if (g2.oin[0] == 1 && g2.oout[0] == 1) {
    RegPassArgs<T> b = a;
    b.g = g2;
    b.in = in;
    b.out = out;
    b.levels = levels;
    b.in_place = false;
    const int rc = launch_col<T>(b, stream, stats, false);
    if (rc != 0) return rc;
  }
  const int rc = launch_whole<T>(a, g2, in, out, levels, true, stream, stats);
  if (rc != 0 || !(g2.oin[0] == 1 && g2.oout[0] == 1)) return rc;
  RegPassArgs<T> b = a;
  b.g = g2;
  b.in = in;
  b.out = out;
  b.levels = levels;
  b.in_place = false;
  return launch_col<T>(b, stream, stats, true);
}

}  // namespace

int check_col_errors(cudaStream_t stream) {
  int32_t* f = col_error_flag();
  if (!f) return 0;
  int32_t v = 0;
  if (cudaStreamSynchronize(stream) != cudaSuccess ||
      cudaMemcpy(&v, f, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  if (v) cudaMemset(f, 0, sizeof(int32_t));
  return v;
}

template <typename T>
int plan_reg_pass(const RegPassArgs<T>& a, cudaStream_t stream,
                  RegStats* stats) {
  // Zero, and Constant / Symmetric / Reflect with exact band edges on the
  // kernels built on the register step code (the strided TMA-staged kernel,
  // the whole-line and tiled register kernels)
  if (edge_footprint(*a.prog, a.bc) < 0) return 0;
  const bool zero = a.bc == BC_ZERO;
  if (a.wi < 0 || a.wi >= kNumCatalogue) return 0;
  // the edge work is compiled into the per-wavelet kernels only
  if (!zero && !compiled_wavelet(a.wi)) return 0;
  if (a.levels < 1 || a.levels > MAX_LEVELS) return 0;
  if (!structure_matches(*a.prog, a.wi, a.op)) return 0;
  const LineGeom& g = a.g;
  if (edges_overlap(*a.prog, g.n, a.levels)) return 0;
  const bool contiguous = (g.sin == 1 && g.sout == 1);
  if (!compiled_wavelet(a.wi)) {
    // the generic instantiations: rows of 512-4096 (float32) or 512-2048
    // (float64) samples, strided lines adjacent in memory
    if (!generic_enabled()) return 0;
    if (contiguous) {
      if (!zero) return 0;
      const int rc = launch_wrow<T>(a, stream, stats);
      if (rc != 0) return rc;
      return launch_wtile<T>(a, stream, stats);
    }
    if (lines_adjacent(g)) return launch_col<T>(a, stream, stats, true);
    return 0;
  }
  // whole lines: contiguous rows, or strided lines adjacent in memory
  if (contiguous) {
    int rc = launch_wrow<T>(a, stream, stats);
    if (rc != 0) return rc;
    if (zero) {
      rc = launch_wtile<T>(a, stream, stats);
      if (rc != 0) return rc;
    }
    rc = launch_whole<T>(a, g, a.in, a.out, a.levels, false, stream, stats);
    if (rc != 0) return rc;
  }
  if (lines_adjacent(g)) {
    // the TMA-staged form first, then the register kernels (plain loads,
    // with their prefetch), then the plain-load form of the strided kernel
    int rc = launch_col<T>(a, stream, stats, false);
    if (rc != 0) return rc;
    rc = launch_whole<T>(a, g, a.in, a.out, a.levels, true, stream, stats);
    if (rc != 0) return rc;
    rc = launch_tiled<T>(a, stream, stats);
    if (rc != 0) return rc;
    return launch_col<T>(a, stream, stats, true);
  }
  return 0;
}

template int plan_reg_pass<float>(const RegPassArgs<float>&, cudaStream_t,
                                  RegStats*);
template int plan_reg_pass<double>(const RegPassArgs<double>&, cudaStream_t,
                                   RegStats*);

}  // namespace lw
