// General exact line kernel of the B200 lifting DWT.
//
// One CTA transforms a batch of W whole lines of one axis pass through every
// level.  The lines live in shared memory (lines up to ~38K float / ~19K
// double) or, for longer lines, in a per-CTA slice of global scratch that
// the caller allocates.  Each lifting step is one parallel pass over the
// updated band, separated by block barriers; the adjoint boundary folds run
// on one thread per line in the reference's order.  The step program is
// interpreted from a by-value parameter, so this one kernel covers every
// catalogue wavelet, user step program, boundary condition and transform.
//
// Semantics restated (paths relative to the jcapriot/lifted tree):
//   boundary index maps            src/lifted-common.hpp:719-779
//   Step<Generic|Unit|Repeat>      src/lifted-steps-inl.hpp:500-615,
//                                  754-885, 1011-1126 (Across form)
//   Step<Scale>                    src/lifted-steps-inl.hpp:1178-1203
//   forward-stepping driver        src/lifted-drivers-inl.hpp:75-142
//   reverse-stepping driver        src/lifted-drivers-inl.hpp:182-274
//   (de)interleave                 src/lifted-ops-inl.hpp:80-188
#pragma once

#include <cstdint>

#include "lw_pdl.hpp"
#include "lw_types.hpp"

namespace lw {

__device__ __forceinline__ float fop(int sub, float v, float x, float y) {
  return sub ? __fmaf_rn(-v, x, y) : __fmaf_rn(v, x, y);
}
__device__ __forceinline__ double fop(int sub, double v, double x, double y) {
  return sub ? __fma_rn(-v, x, y) : __fma_rn(v, x, y);
}

// Boundary index map; returns n for "skip this tap".  Periodic is i % n with
// i taken as an unsigned 64-bit value (the reference's ptrdiff_t % size_t),
// a true wrap only for power-of-two n.  The host never launches inputs on
// which the reference's Symmetric/Reflect loops do not terminate; the
// iteration cap only guarantees that the device cannot spin.
__device__ __forceinline__ uint64_t bc_index(int bc, int64_t i, int64_t n) {
  switch (bc) {
    case BC_ZERO:
      return (i < 0 || i >= n) ? (uint64_t)n : (uint64_t)i;
    case BC_CONSTANT:
      if (i < 0) return 0;
      if (i >= n) return (uint64_t)(n - 1);
      return (uint64_t)i;
    case BC_PERIODIC:
      return n > 0 ? (uint64_t)i % (uint64_t)n : (uint64_t)n;
    case BC_SYMMETRIC: {
      int64_t io = i;
      for (int it = 0; it < 4096 && (io >= n || io < 0); ++it)
        io = io < 0 ? -(io + 1) : 2 * (n - 1) - (io - 1);
      return (io >= n || io < 0) ? (uint64_t)n : (uint64_t)io;
    }
    default: {  // BC_REFLECT
      int64_t io = i;
      for (int it = 0; it < 4096 && (io >= n || io < 0); ++it)
        io = io < 0 ? -io : 2 * (n - 1) - io;
      return (io >= n || io < 0) ? (uint64_t)n : (uint64_t)io;
    }
  }
}

// y updated at index i from band x (length nx) with boundary map bc:
// ip::inner_product (src/lifted-steps-inl.hpp:163-211), unit steps
// (:813-820).  With every tap in range this equals the interior form.
template <typename T>
__device__ __forceinline__ T ip_bc(const DevStep<T>& st, int bc, T y,
                                   const T* x, int64_t nx, int64_t i) {
  const int64_t io = i + st.off;
  if (st.kind == K_GEN) {
    for (int k = 0; k < st.ntaps; ++k) {
      uint64_t ib = bc_index(bc, io + k, nx);
      if (ib < (uint64_t)nx) y = fop(st.sub, st.c[k], x[ib], y);
    }
  } else if (st.kind == K_REPEAT) {
    uint64_t ib = bc_index(bc, io, nx);
    T x0 = ib < (uint64_t)nx ? x[ib] : T(0);
    for (int k = 1; k < st.ntaps; ++k) {
      ib = bc_index(bc, io + k, nx);
      if (ib < (uint64_t)nx) x0 += x[ib];
    }
    y = fop(st.sub, st.c[0], x0, y);
  } else {  // unit
    uint64_t ib = bc_index(bc, io, nx);
    if (ib < (uint64_t)nx) y = st.sub ? y - x[ib] : y + x[ib];
  }
  return y;
}

// Interior form: every tap is known to be in range.
template <typename T>
__device__ __forceinline__ T ip_interior(const DevStep<T>& st, T y,
                                         const T* x, int64_t i) {
  const T* xp = x + (i + st.off);
  if (st.kind == K_GEN) {
    for (int k = 0; k < st.ntaps; ++k) y = fop(st.sub, st.c[k], xp[k], y);
  } else if (st.kind == K_REPEAT) {
    T x0 = xp[0];
    for (int k = 1; k < st.ntaps; ++k) x0 += xp[k];
    y = fop(st.sub, st.c[0], x0, y);
  } else {
    y = st.sub ? y - xp[0] : y + xp[0];
  }
  return y;
}

// ip::inner_product_safe (src/lifted-steps-inl.hpp:330-371): taps from
// x-index j, dropped outside [0, nx).
template <typename T>
__device__ __forceinline__ T ip_safe(const DevStep<T>& st, T y, const T* x,
                                     int64_t j, int64_t nx) {
  if (st.kind == K_GEN) {
    for (int k = 0; k < st.ntaps; ++k) {
      int64_t ii = j + k;
      if (ii >= 0 && ii < nx) y = fop(st.sub, st.c[k], x[ii], y);
    }
  } else {  // repeat
    T x0 = (j >= 0 && j < nx) ? x[j] : T(0);
    for (int k = 1; k < st.ntaps; ++k) {
      int64_t ii = j + k;
      if (ii >= 0 && ii < nx) x0 += x[ii];
    }
    y = fop(st.sub, st.c[0], x0, y);
  }
  return y;
}

// Adjoint front fold of one line (src/lifted-steps-inl.hpp:529-546,
// 781-799, 1041-1058).
template <typename T>
__device__ void fold_front(const DevStep<T>& st, int bc, T* y, int64_t ny,
                           const T* x, int64_t nx) {
  if (st.kind == K_UNIT) {
    for (int64_t i = st.fold_off, j = 0; i < 0 && j < nx; ++i, ++j) {
      uint64_t io = bc_index(bc, i, ny);
      if (io < (uint64_t)ny && (int64_t)io != i)
        y[io] = st.sub ? y[io] - x[j] : y[io] + x[j];
    }
  } else {
    for (int64_t i = st.fold_off, j = 1 - st.ntaps; i < 0; ++i, ++j) {
      uint64_t io = bc_index(bc, i, ny);
      if (io < (uint64_t)ny && (int64_t)io != i)
        y[io] = ip_safe(st, y[io], x, j, nx);
    }
  }
}

// Adjoint back fold of one line (src/lifted-steps-inl.hpp:576-593,
// 838-855, 1088-1104).  i runs from nd (not ny) in the reference.
template <typename T>
__device__ void fold_back(const DevStep<T>& st, int bc, T* y, int64_t ny,
                          const T* x, int64_t nx, int64_t nd) {
  for (int64_t i = nd, j = nd + st.off; i < nx - st.off; ++i, ++j) {
    uint64_t io = bc_index(bc, i, ny);
    if (io < (uint64_t)ny && (int64_t)io != i) {
      if (st.kind == K_UNIT) {
        if (j >= 0 && j < nx) y[io] = st.sub ? y[io] - x[j] : y[io] + x[j];
      } else {
        y[io] = ip_safe(st, y[io], x, j, nx);
      }
    }
  }
}

// Line j and position i of flat index f over W lines of m elements (no
// division for a single line).  Several lines are only ever held in shared
// memory (W * m < 2^31), so a 32-bit division serves them.
__device__ __forceinline__ void split_index(int64_t f, int64_t m, int W, int& j, int64_t& i) {
  if (W == 1) {
    j = 0;
    i = f;
  } else {
    const uint32_t q = (uint32_t)f / (uint32_t)m;
    j = (int)q;
    i = f - (int64_t)q * m;
  }
}

// Line j and position i of flat index f over W lines of n elements, walking
// the positions fastest (contiguous lines) or the lines fastest (strided
// lines, adjacent in memory); 32-bit division as in split_index.
__device__ __forceinline__ void line_pos(int64_t f, int64_t n, int W, bool lines_fastest, int& j,
                                         int64_t& i) {
  if (W == 1) {
    j = 0;
    i = f;
  } else if (lines_fastest) {
    const uint32_t q = (uint32_t)f / (uint32_t)W;
    i = q;
    j = (int)((uint32_t)f - q * (uint32_t)W);
  } else {
    const uint32_t q = (uint32_t)f / (uint32_t)n;
    j = (int)q;
    i = f - (int64_t)q * n;
  }
}

// One step over W lines held at A + j * pitch as [s (ns) | d (nd)].
template <typename T>
__device__ void run_step(const DevStep<T>& st, int normal, int across,
                         int bc, T* A, int64_t pitch, int W, int64_t ns,
                         int64_t nd) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  if (st.kind == K_SCALE) {
    const int64_t m = ns + nd;
    const int64_t tot = (int64_t)W * m;
    for (int64_t f = tid; f < tot; f += nth) {
      int j;
      int64_t i;
      split_index(f, m, W, j, i);
      T* p = A + j * pitch + i;
      *p = *p * (i < ns ? st.sm : st.dm);
    }
    __syncthreads();
    return;
  }
  const int64_t nx = st.y_is_d ? ns : nd;
  const int64_t ny = st.y_is_d ? nd : ns;
  const int64_t xo = st.y_is_d ? 0 : ns;
  const int64_t yo = st.y_is_d ? ns : 0;
  const int64_t n1 = st.nf < ny ? (int64_t)st.nf : ny;
  const int64_t n2 = nd > st.nb ? nd - st.nb : 0;
  if (normal) {
    // front [0,n1) and back [n2,ny) with the boundary map, interior between;
    // indices in both edge ranges get both updates, front first (Q5).
    const int64_t tot = (int64_t)W * ny;
    for (int64_t f = tid; f < tot; f += nth) {
      int j;
      int64_t i;
      split_index(f, ny, W, j, i);
      T* line = A + j * pitch;
      const T* x = line + xo;
      T y = line[yo + i];
      if (i < n1) y = ip_bc(st, bc, y, x, nx, i);
      if (i >= n1 && i < n2) y = ip_interior(st, y, x, i);
      if (i >= n2) y = ip_bc(st, bc, y, x, nx, i);
      line[yo + i] = y;
    }
    __syncthreads();
    return;
  }
  // adjoint: front fold, front+interior direct, then the back fold and the
  // back direct loop in the selected order.
  for (int j = tid; j < W; j += nth) {
    T* line = A + j * pitch;
    fold_front(st, bc, line + yo, ny, line + xo, nx);
  }
  __syncthreads();
  {
    int64_t hi = n1 > n2 ? n1 : n2;
    if (hi > ny) hi = ny;
    if (hi > 0) {
      const int64_t tot = (int64_t)W * hi;
      for (int64_t f = tid; f < tot; f += nth) {
        int j;
        int64_t i;
        split_index(f, hi, W, j, i);
        T* line = A + j * pitch;
        const T* x = line + xo;
        T y = line[yo + i];
        if (i < n1) y = ip_bc(st, BC_ZERO, y, x, nx, i);
        else y = ip_interior(st, y, x, i);
        line[yo + i] = y;
      }
    }
  }
  __syncthreads();
  const int64_t nback = ny > n2 ? ny - n2 : 0;
  for (int pass = 0; pass < 2; ++pass) {
    const bool do_fold = (pass == (across ? 0 : 1));
    if (do_fold) {
      for (int j = tid; j < W; j += nth) {
        T* line = A + j * pitch;
        fold_back(st, bc, line + yo, ny, line + xo, nx, nd);
      }
    } else if (nback > 0) {
      const int64_t tot = (int64_t)W * nback;
      for (int64_t f = tid; f < tot; f += nth) {
        int j;
        int64_t i;
        split_index(f, nback, W, j, i);
        i += n2;
        T* line = A + j * pitch;
        line[yo + i] = ip_bc(st, BC_ZERO, line[yo + i], line + xo, nx, i);
      }
    }
    __syncthreads();
  }
}

template <typename T>
__device__ __forceinline__ void run_program(const DevProgram<T>& prog, int bc,
                                            T* A, int64_t pitch, int W,
                                            int64_t ns, int64_t nd) {
  for (int k = 0; k < prog.nsteps; ++k)
    run_step(prog.st[k], prog.normal, prog.across, bc, A, pitch, W, ns, nd);
}

// One step over W lines held as in run_step, Zero boundary, on bands where
// no step's front edge range [0, n1) reaches past the start n2 of its back
// edge range (the host checks every level: zero_fast_ok).  There run_step
// gives every index of y one update, whose sum runs over the taps inside the
// source band in tap order (the front and back loops through the Zero map,
// which drops the others; the interior loop, whose taps are all inside), in
// both directions: the Zero boundary's adjoint folds change nothing.  This
// computes that sum directly, without the boundary map or the partition.
template <typename T>
__device__ void zero_step(const DevStep<T>& st, T* A, int64_t pitch, int W,
                          int64_t ns, int64_t nd) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  if (st.kind == K_SCALE) {
    const int64_t m = ns + nd;
    const int64_t tot = (int64_t)W * m;
    for (int64_t f = tid; f < tot; f += nth) {
      int j;
      int64_t i;
      split_index(f, m, W, j, i);
      T* p = A + j * pitch + i;
      *p = *p * (i < ns ? st.sm : st.dm);
    }
    return;
  }
  const int64_t nx = st.y_is_d ? ns : nd;
  const int64_t ny = st.y_is_d ? nd : ns;
  const int64_t xo = st.y_is_d ? 0 : ns;
  const int64_t yo = st.y_is_d ? ns : 0;
  const int64_t tot = (int64_t)W * ny;
  if (tot <= 0x7fffffffLL && nx + st.ntaps <= 0x7fffffffLL) {
    // 32-bit positions (every shared-memory batch of lines, and any line
    // shorter than 2^31)
    const int nx32 = (int)nx, ny32 = (int)ny, tot32 = (int)tot;
    for (int f = tid; f < tot32; f += nth) {
      const int j = W == 1 ? 0 : (int)((unsigned)f / (unsigned)ny32);
      const int i = f - j * ny32;
      T* line = A + j * pitch;
      const T* x = line + xo;
      const int b = i + st.off;
      T y = line[yo + i];
      if (st.kind == K_UNIT) {
        if (b >= 0 && b < nx32) y = st.sub ? y - x[b] : y + x[b];
      } else if (b >= 0 && b + st.ntaps <= nx32) {
        y = ip_interior(st, y, x, i);
      } else {
        y = ip_safe(st, y, x, b, nx);
      }
      line[yo + i] = y;
    }
    return;
  }
  for (int64_t f = tid; f < tot; f += nth) {
    int j;
    int64_t i;
    split_index(f, ny, W, j, i);
    T* line = A + j * pitch;
    const T* x = line + xo;
    const int64_t b = i + st.off;
    T y = line[yo + i];
    if (st.kind == K_UNIT) {
      if (b >= 0 && b < nx) y = st.sub ? y - x[b] : y + x[b];
    } else if (b >= 0 && b + st.ntaps <= nx) {
      y = ip_interior(st, y, x, i);
    } else {
      y = ip_safe(st, y, x, b, nx);
    }
    line[yo + i] = y;
  }
}

// The step program on W lines: the exact step code, or (zf) zero_step.
template <typename T>
__device__ __forceinline__ void run_program_sel(const DevProgram<T>& prog, int bc, bool zf,
                                                T* A, int64_t pitch, int W,
                                                int64_t ns, int64_t nd) {
  if (!zf) {
    run_program(prog, bc, A, pitch, W, ns, nd);
    return;
  }
  for (int k = 0; k < prog.nsteps; ++k) {
    zero_step(prog.st[k], A, pitch, W, ns, nd);
    __syncthreads();
  }
}

// Forward-stepping levels on W lines held raw (not yet split) at
// A + j * pitch, length m each (B needs m elements per line): every level splits A[0..m) into
// [evens | odds] through B (src/lifted-ops-inl.hpp:104-135), runs the steps
// and recurses on the evens (src/lifted-drivers-inl.hpp:117-139).  On return
// A[0..m) holds [a | d_last | ... | d_first] of these levels.
template <typename T>
__device__ void coarse_forward(const DevProgram<T>& prog, int bc, T* A,
                               int64_t pitch, T* B, int64_t pitch_b, int W,
                               int64_t m, int nlev, bool zf = false) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  for (int lvl = 0; lvl < nlev; ++lvl) {
    const int64_t nd = m / 2, ns = m - nd;
    const int64_t t2 = (int64_t)W * m;
    for (int64_t f = tid; f < t2; f += nth) {
      int j;
      int64_t i;
      split_index(f, m, W, j, i);
      B[j * pitch_b + i] = A[j * pitch + i];
    }
    __syncthreads();
    for (int64_t f = tid; f < t2; f += nth) {
      int j;
      int64_t i;
      split_index(f, m, W, j, i);
      A[j * pitch + ((i & 1) ? ns + (i >> 1) : (i >> 1))] = B[j * pitch_b + i];
    }
    __syncthreads();
    run_program_sel(prog, bc, zf, A, pitch, W, ns, nd);
    m = ns;
  }
}

// Reverse-stepping levels on W lines (B needs m0 elements per line):
// A[0..m0) holds
// [a | d_last | ... | d_first] of `nlev` levels of a line of length m0; each
// level runs the (reversed) steps and interleaves s|d through B
// (src/lifted-drivers-inl.hpp:226-255).  On return A[0..m0) is the line.
template <typename T>
__device__ void coarse_reverse(const DevProgram<T>& prog, int bc, T* A,
                               int64_t pitch, T* B, int64_t pitch_b, int W,
                               int64_t m0, int nlev, bool zf = false) {
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  int64_t msz[MAX_LEVELS + 1];
  msz[0] = m0;
  for (int l = 1; l <= nlev; ++l) msz[l] = msz[l - 1] - msz[l - 1] / 2;
  for (int lvl = nlev - 1; lvl >= 0; --lvl) {
    const int64_t m = msz[lvl];
    const int64_t nd = m / 2, ns = m - nd;
    run_program_sel(prog, bc, zf, A, pitch, W, ns, nd);
    const int64_t t2 = (int64_t)W * m;
    for (int64_t f = tid; f < t2; f += nth) {
      int j;
      int64_t i;
      split_index(f, m, W, j, i);
      B[j * pitch_b + i] = A[j * pitch + i];
    }
    __syncthreads();
    for (int64_t f = tid; f < t2; f += nth) {
      int j;
      int64_t i;
      split_index(f, m, W, j, i);
      int64_t src = (i & 1) ? ns + (i >> 1) : (i >> 1);
      A[j * pitch + i] = B[j * pitch_b + src];
    }
    __syncthreads();
  }
}

// Base offsets of line `li` in the source and destination.
__device__ __forceinline__ void line_base(const LineGeom& g, int64_t li,
                                          int64_t& bin, int64_t& bout) {
  int64_t r = li;
  bin = 0;
  bout = 0;
  for (int d = 0; d < g.nother; ++d) {
    int64_t q = r / g.oshape[d];
    int64_t idx = r - q * g.oshape[d];
    r = q;
    bin += idx * g.oin[d];
    bout += idx * g.oout[d];
  }
}

template <typename T>
__global__ void __launch_bounds__(512)
    line_kernel(const __grid_constant__ LineParams<T> p) {
  extern __shared__ __align__(16) unsigned char lw_smem_raw[];
  pdl_wait();  // the previous kernel's results (no global access before)
  pdl_trigger();
  __shared__ int64_t s_bin[64];
  __shared__ int64_t s_bout[64];
  const LineGeom& g = p.g;
  const int W = p.W;
  const int64_t n = g.n;
  T* A;
  T* B;
  if (p.use_smem) {
    A = reinterpret_cast<T*>(lw_smem_raw);
  } else {
    A = p.scratch + (int64_t)blockIdx.x * W * (p.pitch + p.pitch_b);
  }
  B = A + (int64_t)W * p.pitch;
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  const bool along_contig = (g.sin == 1 || g.sin == -1);
  const bool along_contig_out = (g.sout == 1 || g.sout == -1);

  for (int64_t first = (int64_t)blockIdx.x * W; first < g.nlines;
       first += p.nlines_per_cta_stride) {
    const int We = (int)((g.nlines - first) < W ? (g.nlines - first) : W);
    for (int j = tid; j < We; j += nth) {
      int64_t bi, bo;
      line_base(g, first + j, bi, bo);
      s_bin[j] = bi;
      s_bout[j] = bo;
    }
    __syncthreads();

    const int64_t tot = (int64_t)We * n;
    if (p.prog.fwd_driver) {
      // Forward-stepping: load deinterleaved ([evens | odds], Q10).
      const int64_t ns0 = n - n / 2;
      for (int64_t f = tid; f < tot; f += nth) {
        int j;
        int64_t i;
        line_pos(f, n, We, !along_contig, j, i);
        T v = p.in[s_bin[j] + i * g.sin];
        A[j * p.pitch + ((i & 1) ? ns0 + (i >> 1) : (i >> 1))] = v;
      }
      __syncthreads();
      int64_t m = n;
      for (int lvl = 0; lvl < p.levels; ++lvl) {
        const int64_t nd = m / 2, ns = m - nd;
        if (lvl > 0) {
          const int64_t t2 = (int64_t)We * m;
          for (int64_t f = tid; f < t2; f += nth) {
            int j;
            int64_t i;
            split_index(f, m, We, j, i);
            B[j * p.pitch_b + i] = A[j * p.pitch + i];
          }
          __syncthreads();
          for (int64_t f = tid; f < t2; f += nth) {
            int j;
            int64_t i;
            split_index(f, m, We, j, i);
            T v = B[j * p.pitch_b + i];
            A[j * p.pitch + ((i & 1) ? ns + (i >> 1) : (i >> 1))] = v;
          }
          __syncthreads();
        }
        run_program_sel(p.prog, p.bc, p.zfast != 0, A, p.pitch, We, ns, nd);
        m = ns;
      }
      // A now holds [a_L | d_L | ... | d_1] (Q11).
      for (int64_t f = tid; f < tot; f += nth) {
        int j;
        int64_t i;
        line_pos(f, n, We, !along_contig_out, j, i);
        p.out[s_bout[j] + i * g.sout] = A[j * p.pitch + i];
      }
    } else {
      // Reverse-stepping: the input is already [a_L | d_L | ... | d_1].
      for (int64_t f = tid; f < tot; f += nth) {
        int j;
        int64_t i;
        line_pos(f, n, We, !along_contig, j, i);
        A[j * p.pitch + i] = p.in[s_bin[j] + i * g.sin];
      }
      __syncthreads();
      int64_t msz[MAX_LEVELS + 1];
      msz[0] = n;
      for (int l = 1; l <= p.levels; ++l) msz[l] = msz[l - 1] - msz[l - 1] / 2;
      for (int lvl = p.levels - 1; lvl >= 0; --lvl) {
        const int64_t m = msz[lvl];
        const int64_t nd = m / 2, ns = m - nd;
        run_program_sel(p.prog, p.bc, p.zfast != 0, A, p.pitch, We, ns, nd);
        if (lvl > 0) {
          const int64_t t2 = (int64_t)We * m;
          for (int64_t f = tid; f < t2; f += nth) {
            int j;
            int64_t i;
            split_index(f, m, We, j, i);
            B[j * p.pitch_b + i] = A[j * p.pitch + i];
          }
          __syncthreads();
          for (int64_t f = tid; f < t2; f += nth) {
            int j;
            int64_t i;
            split_index(f, m, We, j, i);  // output index
            int64_t src = (i & 1) ? ns + (i >> 1) : (i >> 1);
            A[j * p.pitch + i] = B[j * p.pitch_b + src];
          }
          __syncthreads();
        }
      }
      // Level 0 interleaves straight into the destination.
      const int64_t ns0 = n - n / 2;
      for (int64_t f = tid; f < tot; f += nth) {
        int j;
        int64_t i;
        line_pos(f, n, We, !along_contig_out, j, i);
        int64_t src = (i & 1) ? ns0 + (i >> 1) : (i >> 1);
        p.out[s_bout[j] + i * g.sout] = A[j * p.pitch + src];
      }
    }
    __syncthreads();
  }
}

}  // namespace lw
