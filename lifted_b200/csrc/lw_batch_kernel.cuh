// Persistent batch kernel of the B200 lifting DWT: many uneven 1D signals,
// each with its own wavelet and level count, in one launch (work items and
// their meaning: lw_batch.hpp).
//
// Every CTA loops: take the next item index from the device queue (one
// atomic), copy the item's step program to shared memory, wait (bounded) for
// the producer group of its input band if it has one, run the item, and
// publish completion (barrier, fence, atomic increment).  Items run in
// shared memory; a tile item holds its window as split s/d halves and runs
// one parallel pass per lifting step.
//
// Tile arithmetic is the Zero-boundary per-element form of the reference's
// steps (src/lifted-steps-inl.hpp:163-211, 813-820, 1011-1126): taps
// outside the band are skipped, generic steps are sequential fused
// multiply-adds, repeat steps sum their taps first, unit steps add or
// subtract.  With the Zero boundary the adjoint folds never write
// (src/lifted-steps-inl.hpp:529-546, 576-593), and on bands long enough for
// tiles the front, interior and back loops give each element exactly this
// form.  Whole items run the general exact step code of the line kernel.
#pragma once

#include <cstddef>
#include <cstdint>

#include "lw_batch.hpp"
#include "lw_line_kernel.cuh"

namespace lw {
namespace batch {

__device__ __forceinline__ int32_t ld_acquire(const int32_t* p) {
  int32_t v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Asynchronous 4- or 8-byte copy global -> shared (cp.async, cached in L1:
// the caller's input is read-only for the launch, and scratch bands start on
// 128-byte boundaries and are complete before any item reads them, so no L1
// line ever holds a value older than the band it belongs to).  Every thread
// issues its copies without waiting; cp_wait() drains them.
template <typename T>
__device__ __forceinline__ void cp_elem(T* sdst, const T* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Length of the band after `l` levels (src/lifted-drivers-inl.hpp:117-139:
// the approximation of a band of m samples has m - m/2).
__device__ __forceinline__ int64_t band_len(int64_t n, int l) {
  for (int i = 0; i < l; ++i) n -= n / 2;
  return n;
}

// Loads of a band: scratch bands are produced by other CTAs of this launch,
// so they bypass L1; the caller's input is read-only for the launch.
template <typename T>
__device__ __forceinline__ T ld_band(int sel, const T* p) {
  return sel == BS_SCRATCH ? __ldcg(p) : __ldg(p);
}

template <typename T>
__device__ __forceinline__ const T* band_ptr(const BatchParams<T>& p, int sel,
                                             int64_t off) {
  return (sel == BS_IN ? p.in : (sel == BS_OUT ? p.out : p.scratch)) + off;
}
template <typename T>
__device__ __forceinline__ T* band_ptr_w(const BatchParams<T>& p, int sel,
                                         int64_t off) {
  return (sel == BS_OUT ? p.out : p.scratch) + off;
}

// One step on a window of the split bands, Zero boundary.  Window element q
// of S and D is global pair gb + q; nsw / ndw are the window's s and d
// counts, ns / nd the band's.  A tap at window index i counts when
// 0 <= i < min(window count, band length - gb): below 0 it lies before the
// window (outside the band, or in the corrupted margin the halo absorbs),
// beyond it after the window or the band.
template <typename T>
__device__ __forceinline__ void tile_step(const DevStep<T>& st, T* S, T* D,
                                          int64_t gb, int nsw, int ndw,
                                          int64_t ns, int64_t nd) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  if (st.kind == K_SCALE) {
    const T sm = st.sm, dm = st.dm;
    for (int q = tid; q < nsw; q += nth) S[q] = S[q] * sm;
    for (int q = tid; q < ndw; q += nth) D[q] = D[q] * dm;
    return;
  }
  T* Y = st.y_is_d ? D : S;
  const T* X = st.y_is_d ? S : D;
  const int nyw = st.y_is_d ? ndw : nsw;
  const int nxw = st.y_is_d ? nsw : ndw;
  const int64_t nxg = (st.y_is_d ? ns : nd) - gb;
  const int xhi = (int)(nxg < (int64_t)nxw ? nxg : (int64_t)nxw);
  const int off = st.off, nt = st.ntaps, sub = st.sub;
  if (st.kind == K_GEN && nt <= 2) {
    const T c0 = sub ? -st.c[0] : st.c[0];
    const T c1 = sub ? -st.c[1] : st.c[1];
    for (int q = tid; q < nyw; q += nth) {
      const int b = q + off;
      T y = Y[q];
      if (b >= 0 && b + nt <= xhi) {
        y = fop(0, c0, X[b], y);
        if (nt == 2) y = fop(0, c1, X[b + 1], y);
      } else {
        if (b >= 0 && b < xhi) y = fop(0, c0, X[b], y);
        if (nt == 2 && b + 1 >= 0 && b + 1 < xhi) y = fop(0, c1, X[b + 1], y);
      }
      Y[q] = y;
    }
  } else if (st.kind == K_GEN) {
    for (int q = tid; q < nyw; q += nth) {
      const int b = q + off;
      T y = Y[q];
      if (b >= 0 && b + nt <= xhi) {
        for (int k = 0; k < nt; ++k) y = fop(sub, st.c[k], X[b + k], y);
      } else {
        for (int k = 0; k < nt; ++k) {
          const int i = b + k;
          if (i >= 0 && i < xhi) y = fop(sub, st.c[k], X[i], y);
        }
      }
      Y[q] = y;
    }
  } else if (st.kind == K_REPEAT && nt == 2) {
    const T c0 = sub ? -st.c[0] : st.c[0];
    for (int q = tid; q < nyw; q += nth) {
      const int b = q + off;
      T x0;
      if (b >= 0 && b + 2 <= xhi) {
        x0 = X[b] + X[b + 1];
      } else {
        x0 = (b >= 0 && b < xhi) ? X[b] : T(0);
        if (b + 1 >= 0 && b + 1 < xhi) x0 += X[b + 1];
      }
      Y[q] = fop(0, c0, x0, Y[q]);
    }
  } else if (st.kind == K_REPEAT) {
    for (int q = tid; q < nyw; q += nth) {
      const int b = q + off;
      T x0;
      if (b >= 0 && b + nt <= xhi) {
        x0 = X[b];
        for (int k = 1; k < nt; ++k) x0 += X[b + k];
      } else {
        x0 = (b >= 0 && b < xhi) ? X[b] : T(0);
        for (int k = 1; k < nt; ++k) {
          const int i = b + k;
          if (i >= 0 && i < xhi) x0 += X[i];
        }
      }
      Y[q] = fop(sub, st.c[0], x0, Y[q]);
    }
  } else {  // unit
    for (int q = tid; q < nyw; q += nth) {
      const int i = q + off;
      if (i >= 0 && i < xhi) Y[q] = sub ? Y[q] - X[i] : Y[q] + X[i];
    }
  }
}

template <typename T>
__device__ __forceinline__ void tile_program(const DevProgram<T>& prog, T* S,
                                             T* D, int64_t gb, int nsw,
                                             int ndw, int64_t ns, int64_t nd) {
  for (int k = 0; k < prog.nsteps; ++k) {
    tile_step(prog.st[k], S, D, gb, nsw, ndw, ns, nd);
    __syncthreads();
  }
}

// Forward-stepping tile: levels lev0+1 .. lev0+nlev of band lev0 on the
// window [t0 - halo, t1 + halo); stores the interior of every detail band
// (to its place in the output layout [a_L | d_L | ... | d_1]) and of the
// last approximation band.  buf: 3 * cap2 elements.
template <typename T>
__device__ void tile_fwd(const BatchParams<T>& p, const BatchItem& w,
                         const DevProgram<T>& prog, T* buf, int64_t cap2) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  int64_t m = band_len(w.n0, w.lev0);
  const T* src = band_ptr(p, w.src_sel, w.src_off);
  int64_t wl0 = w.t0 - w.halo;
  if (wl0 < 0) wl0 = 0;
  int64_t wl1 = w.t1 + w.halo;
  if (wl1 > m) wl1 = m;
  T* S = buf;
  T* D = buf + cap2;
  T* X = buf + 2 * cap2;
  {
    const int cnt = (int)(wl1 - wl0);
    const T* s0 = src + wl0;
    for (int i = tid; i < cnt; i += nth) cp_elem((i & 1) ? D + (i >> 1) : S + (i >> 1), s0 + i);
    cp_wait();
  }
  __syncthreads();
  int64_t il0 = w.t0;
  int64_t il1 = w.t1 < m ? w.t1 : m;
  for (int j = 0; j < w.nlev; ++j) {
    const int64_t nd = m / 2, ns = m - nd;
    const int64_t gb = wl0 >> 1;
    const int nsw = (int)((wl1 - wl0 + 1) >> 1);
    const int ndw = (int)((wl1 - wl0) >> 1);
    tile_program(prog, S, D, gb, nsw, ndw, ns, nd);
    // d of level lev0+j+1 sits at [ns, m) of this band's output region
    T* dout = p.out + w.out_off + ns;
    const int64_t d_lo = il0 >> 1, d_hi = il1 >> 1;
    for (int64_t q = d_lo + tid; q < d_hi; q += nth) dout[q] = D[q - gb];
    il0 >>= 1;
    il1 = (il1 + 1) >> 1;
    wl0 = gb;
    wl1 = gb + nsw;
    m = ns;
    if (j + 1 < w.nlev) {
      // split the approximation band in one pass: evens to X, odds to D
      // (D was stored above), then X becomes S
      __syncthreads();
      for (int i = tid; i < nsw; i += nth) {
        const T v = S[i];
        if (i & 1) D[i >> 1] = v;
        else X[i >> 1] = v;
      }
      __syncthreads();
      T* t = S;
      S = X;
      X = t;
    }
  }
  T* dst = band_ptr_w(p, w.dst_sel, w.dst_off);
  for (int64_t q = il0 + tid; q < il1; q += nth) dst[q] = S[q - wl0];
}

// Reverse-stepping tile: from the approximation band of level lev0+nlev and
// the detail bands d_{lev0+nlev} .. d_{lev0+1} (read from the coefficient
// layout of the input) back to band lev0, on the window
// [t0 - halo, t1 + halo) of band lev0; stores the interior [t0, t1).
template <typename T>
__device__ void tile_rev(const BatchParams<T>& p, const BatchItem& w,
                         const DevProgram<T>& prog, T* buf, int64_t cap2) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  int64_t mlev[MAX_LEVELS + 1];
  int64_t wl1[MAX_LEVELS + 1];
  mlev[0] = band_len(w.n0, w.lev0);
  int64_t W0 = w.t0 - w.halo;
  if (W0 < 0) W0 = 0;
  wl1[0] = w.t1 + w.halo;
  if (wl1[0] > mlev[0]) wl1[0] = mlev[0];
  for (int j = 0; j < w.nlev; ++j) {
    mlev[j + 1] = mlev[j] - mlev[j] / 2;
    wl1[j + 1] = (wl1[j] + 1) >> 1;
  }
  T* S = buf;
  T* D = buf + cap2;
  T* X = buf + 2 * cap2;
  const T* dsrc = p.in + w.in_off;
  {
    // approximation band of level lev0+nlev: window pairs of level nlev-1
    const int j = w.nlev - 1;
    const int64_t gb = (W0 >> j) >> 1;
    const int nsw = (int)(wl1[j + 1] - gb);
    const T* src = band_ptr(p, w.src_sel, w.src_off) + gb;
    for (int q = tid; q < nsw; q += nth) cp_elem(S + q, src + q);
  }
  for (int j = w.nlev - 1; j >= 0; --j) {
    const int64_t m = mlev[j];
    const int64_t ns = mlev[j + 1], nd = m - ns;
    const int64_t wl0 = W0 >> j;
    const int64_t gb = wl0 >> 1;
    const int nsw = (int)((wl1[j] - wl0 + 1) >> 1);
    const int ndw = (int)((wl1[j] - wl0) >> 1);
    {
      // d of level lev0+j+1 at [ns, m) of the coefficient layout
      const T* d0 = dsrc + ns + gb;
      for (int q = tid; q < ndw; q += nth) cp_elem(D + q, d0 + q);
      cp_wait();
    }
    __syncthreads();
    tile_program(prog, S, D, gb, nsw, ndw, ns, nd);
    if (j > 0) {
      const int cnt = (int)(wl1[j] - wl0);
      for (int i = tid; i < cnt; i += nth) X[i] = (i & 1) ? D[i >> 1] : S[i >> 1];
      __syncthreads();
      T* t = S;
      S = X;
      X = t;
    } else {
      T* dst = band_ptr_w(p, w.dst_sel, w.dst_off);
      const int64_t hi = w.t1 < m ? w.t1 : m;
      for (int64_t pos = w.t0 + tid; pos < hi; pos += nth) {
        const int64_t r = pos - wl0;
        dst[pos] = (r & 1) ? D[r >> 1] : S[r >> 1];
      }
    }
  }
}

// Whole forward item: levels lev0+1 .. lev0+nlev of band lev0 with the exact
// general step code; band lev0's output region [0, m) gets
// [a | d_last | ... | d_first] of these levels.
template <typename T>
__device__ void whole_fwd(const BatchParams<T>& p, const BatchItem& w,
                          const DevProgram<T>& prog, T* A, int bc) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  const int64_t m = band_len(w.n0, w.lev0);
  const int64_t nd = m / 2, ns = m - nd;
  T* B = A + m;
  const T* src = band_ptr(p, w.src_sel, w.src_off);
  if (w.gbuf < 0) {
    for (int64_t i = tid; i < m; i += nth) cp_elem(A + ((i & 1) ? ns + (i >> 1) : (i >> 1)), src + i);
    cp_wait();
  } else {
    for (int64_t i = tid; i < m; i += nth)
      A[(i & 1) ? ns + (i >> 1) : (i >> 1)] = ld_band(w.src_sel, src + i);
  }
  __syncthreads();
  run_program_sel(prog, bc, w.zfast != 0, A, m, 1, ns, nd);
  if (w.nlev > 1) coarse_forward(prog, bc, A, m, B, ns, 1, ns, w.nlev - 1, w.zfast != 0);
  T* dst = p.out + w.out_off;
  for (int64_t i = tid; i < m; i += nth) dst[i] = A[i];
}

// Whole reverse item: from [a_L | d_L | ... | d_{lev0+1}] (the first m
// coefficients of the signal) to band lev0.
template <typename T>
__device__ void whole_rev(const BatchParams<T>& p, const BatchItem& w,
                          const DevProgram<T>& prog, T* A, int bc) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  const int64_t m = band_len(w.n0, w.lev0);
  const int64_t nd = m / 2, ns = m - nd;
  T* B = A + m;
  const T* src = p.in + w.in_off;
  if (w.gbuf < 0) {
    for (int64_t i = tid; i < m; i += nth) cp_elem(A + i, src + i);
    cp_wait();
  } else {
    for (int64_t i = tid; i < m; i += nth) A[i] = __ldg(src + i);
  }
  __syncthreads();
  if (w.nlev > 1) coarse_reverse(prog, bc, A, m, B, ns, 1, ns, w.nlev - 1, w.zfast != 0);
  run_program_sel(prog, bc, w.zfast != 0, A, m, 1, ns, nd);
  T* dst = band_ptr_w(p, w.dst_sel, w.dst_off);
  for (int64_t i = tid; i < m; i += nth)
    dst[i] = A[(i & 1) ? ns + (i >> 1) : (i >> 1)];
}

// Element offset of line L of an nD axis pass (BatchAxisGeom).
__device__ __forceinline__ int64_t axis_line_base(const BatchAxisGeom& g, int64_t L) {
  const int64_t i0 = L % g.oshape[0];
  const int64_t r = L / g.oshape[0];
  const int64_t i1 = r % g.oshape[1];
  const int64_t i2 = r / g.oshape[1];
  return i0 * g.ostride[0] + i1 * g.ostride[1] + i2 * g.ostride[2];
}

// Line item, forward-stepping: lines [t0, t1) of an nD image's axis pass,
// every level of the axis, with the exact general step code over W lines at
// once (the line kernel's multi-line form: src/lifted-drivers-inl.hpp:
// 75-142 per line).  A holds the lines (pitch n), B their split buffers.
// The source is `in` for the image's first axis and `out` (in place) for
// the later ones (src/lifted-drivers-inl.hpp:459-485).
// Element offsets of the item's lines (at most kMaxItemLines) in `base`.
constexpr int kMaxItemLines = 64;
__device__ __forceinline__ void item_bases(const BatchItem& w, const BatchAxisGeom& g,
                                           int64_t* base) {
  const int W = (int)(w.t1 - w.t0);
  for (int j = threadIdx.x; j < W; j += blockDim.x) base[j] = axis_line_base(g, w.t0 + j);
  __syncthreads();
}

template <typename T>
__device__ void lines_fwd(const BatchParams<T>& p, const BatchItem& w,
                          const DevProgram<T>& prog, T* A, int bc, int64_t* base) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  const BatchAxisGeom& g = p.geos[w.geo];
  item_bases(w, g, base);
  const int64_t n = w.n0, nd = n / 2, ns = n - nd;
  const int W = (int)(w.t1 - w.t0);
  const bool strided = g.sa != 1;
  const bool smem = w.gbuf == -1;
  T* B = A + (int64_t)W * n;
  const T* src = w.src_sel == BS_IN ? p.in + w.in_off : p.out + w.out_off;
  const int64_t tot = (int64_t)W * n;
  for (int64_t f = tid; f < tot; f += nth) {
    int j;
    int64_t i;
    line_pos(f, n, W, strided, j, i);
    const T* q = src + base[j] + i * g.sa;
    T* d = A + (int64_t)j * n + ((i & 1) ? ns + (i >> 1) : (i >> 1));
    if (smem && w.src_sel == BS_IN) cp_elem(d, q);
    else *d = w.src_sel == BS_IN ? __ldg(q) : __ldcg(q);
  }
  if (smem) cp_wait();
  __syncthreads();
  run_program_sel(prog, bc, w.zfast != 0, A, n, W, ns, nd);
  if (w.nlev > 1) coarse_forward(prog, bc, A, n, B, ns, W, ns, w.nlev - 1, w.zfast != 0);
  T* dst = p.out + w.out_off;
  for (int64_t f = tid; f < tot; f += nth) {
    int j;
    int64_t i;
    line_pos(f, n, W, strided, j, i);
    dst[base[j] + i * g.sa] = A[(int64_t)j * n + i];
  }
}

// Line item, reverse-stepping: from [a_L | d_L | ... | d_1] along each line
// back to the signal domain (src/lifted-drivers-inl.hpp:182-274 per line).
template <typename T>
__device__ void lines_rev(const BatchParams<T>& p, const BatchItem& w,
                          const DevProgram<T>& prog, T* A, int bc, int64_t* base) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  const BatchAxisGeom& g = p.geos[w.geo];
  item_bases(w, g, base);
  const int64_t n = w.n0, nd = n / 2, ns = n - nd;
  const int W = (int)(w.t1 - w.t0);
  const bool strided = g.sa != 1;
  const bool smem = w.gbuf == -1;
  T* B = A + (int64_t)W * n;
  const T* src = w.src_sel == BS_IN ? p.in + w.in_off : p.out + w.out_off;
  const int64_t tot = (int64_t)W * n;
  for (int64_t f = tid; f < tot; f += nth) {
    int j;
    int64_t i;
    line_pos(f, n, W, strided, j, i);
    const T* q = src + base[j] + i * g.sa;
    T* d = A + (int64_t)j * n + i;
    if (smem && w.src_sel == BS_IN) cp_elem(d, q);
    else *d = w.src_sel == BS_IN ? __ldg(q) : __ldcg(q);
  }
  if (smem) cp_wait();
  __syncthreads();
  if (w.nlev > 1) coarse_reverse(prog, bc, A, n, B, ns, W, ns, w.nlev - 1, w.zfast != 0);
  run_program_sel(prog, bc, w.zfast != 0, A, n, W, ns, nd);
  T* dst = p.out + w.out_off;
  for (int64_t f = tid; f < tot; f += nth) {
    int j;
    int64_t i;
    line_pos(f, n, W, strided, j, i);
    dst[base[j] + i * g.sa] = A[(int64_t)j * n + ((i & 1) ? ns + (i >> 1) : (i >> 1))];
  }
}

}  // namespace batch

template <typename T>
__global__ void __launch_bounds__(512)
    batch_kernel(const __grid_constant__ BatchParams<T> p) {
  extern __shared__ __align__(16) unsigned char lw_batch_smem[];
  DevProgram<T>* prog = reinterpret_cast<DevProgram<T>*>(lw_batch_smem);
  T* buf = reinterpret_cast<T*>(lw_batch_smem +
                                ((sizeof(DevProgram<T>) + 15) / 16) * 16);
  __shared__ int32_t s_item;
  __shared__ int32_t s_ok;
  __shared__ int64_t s_base[batch::kMaxItemLines];
  const int64_t cap2 = p.buf_elems / 3;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(p.head, 1);
    __syncthreads();
    const int32_t it = s_item;
    if (it >= p.nitems) break;
    const BatchItem w = p.items[it];
    {
      // the item's program: header and its steps only
      const DevProgram<T>* gp = p.progs + w.prog;
      const int nsteps = gp->nsteps;
      const size_t bytes = offsetof(DevProgram<T>, st) + (size_t)nsteps * sizeof(DevStep<T>);
      const int32_t* s32 = reinterpret_cast<const int32_t*>(gp);
      int32_t* d32 = reinterpret_cast<int32_t*>(prog);
      for (int k = threadIdx.x; k < (int)(bytes / 4); k += blockDim.x) d32[k] = s32[k];
    }
    if (threadIdx.x == 0) {
      int32_t ok = 1;
      if (w.wait_ctr >= 0) {
        ok = 0;
        for (int32_t k = 0; k < p.spin_limit; ++k) {
          if (batch::ld_acquire(p.counters + w.wait_ctr) >= w.wait_target) {
            ok = 1;
            break;
          }
          __nanosleep(200);
        }
        if (!ok) atomicCAS(p.error, 0, it + 1);
      }
      s_ok = ok;
    }
    __syncthreads();
    if (s_ok) {
      T* A = w.gbuf >= 0 ? p.scratch + w.gbuf : buf;
      switch (w.kind) {
        case BI_TILE_FWD:
          batch::tile_fwd(p, w, *prog, buf, cap2);
          break;
        case BI_TILE_REV:
          batch::tile_rev(p, w, *prog, buf, cap2);
          break;
        case BI_WHOLE_FWD:
          batch::whole_fwd(p, w, *prog, A, p.bc);
          break;
        case BI_LINES_FWD:
          batch::lines_fwd(p, w, *prog,
                           w.gbuf == -2 ? p.scratch + p.slot_off + blockIdx.x * p.slot_elems : buf,
                           p.bc, s_base);
          break;
        case BI_LINES_REV:
          batch::lines_rev(p, w, *prog,
                           w.gbuf == -2 ? p.scratch + p.slot_off + blockIdx.x * p.slot_elems : buf,
                           p.bc, s_base);
          break;
        default:
          batch::whole_rev(p, w, *prog, A, p.bc);
          break;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && w.done_ctr >= 0) {
      __threadfence();
      atomicAdd(p.counters + w.done_ctr, 1);
    }
  }
}

}  // namespace lw
