// Exact band edges for the register kernels under the Constant, Symmetric
// and Reflect boundaries.
//
// The register kernels update every element of a band with the Zero form of
// a step: taps outside the band are skipped (src/lifted-steps-inl.hpp:
// 163-211 with ZeroBoundary).  The reference's other boundaries differ from
// that only near the band ends:
//   normal steps (Forward, Inverse)   the elements of the front region
//       [0, n1) and the back region [n2, ny) take their out-of-band taps
//       from the mapped indices (src/lifted-steps-inl.hpp:433-497,
//       552-615; index maps src/lifted-common.hpp:719-779);
//   adjoint steps (ForwardAdjoint, InverseAdjoint)  the direct loops are
//       the Zero form, and the fold loops add the taps of the out-of-band
//       positions onto their mapped in-band targets: the front fold before
//       every direct update, the back fold after the front and interior
//       direct updates and, in the Across form, before the back direct
//       updates (src/lifted-steps-inl.hpp:516-598; Along: after them).
// For these three boundaries every mapped index lies within a few elements
// of the band end it mirrors, so the chunk holding a band's first pairs can
// redo its front edge, and the chunk holding the last pairs its back edge,
// with values it already holds: per step, it keeps the old values of the
// elements a normal step recomputes, applies the fold contributions that
// precede the direct update, lets the Zero update run, then recomputes the
// edge elements of a normal step from the kept values and applies the fold
// contributions that follow.  Each element then sees exactly the
// reference's operations in the reference's order.  The host checks that
// every index these loops touch lies within the edge chunk (edge_footprint
// in lw_reg_kernels.cu); Periodic maps to the far end of the band and is
// not served here.
#pragma once

#include <cstdint>

#include "lw_lanevec.cuh"
#include "lw_line_kernel.cuh"

namespace lw {
namespace edge {

// Largest window (pairs) an edge chunk hands to the edge code at each end.
constexpr int kEdge = 12;

// The edge loops work on windows of E pairs of both bands, copied out of the
// chunk's registers into local arrays: band index i is window element
// i - base.

// ip_bc of the line kernel (taps through the boundary map).
template <typename T, typename VT>
__device__ __forceinline__ VT ip_bc(const DevStep<T>& st, int bc, VT y, const VT* x,
                                    int64_t base, int64_t nx, int64_t i) {
  const int64_t io = i + st.off;
  if (st.kind == K_GEN) {
    for (int k = 0; k < st.ntaps; ++k) {
      const uint64_t ib = bc_index(bc, io + k, nx);
      if (ib < (uint64_t)nx) y = vfop(st.sub, st.c[k], x[(int64_t)ib - base], y);
    }
  } else if (st.kind == K_REPEAT) {
    uint64_t ib = bc_index(bc, io, nx);
    VT x0 = ib < (uint64_t)nx ? x[(int64_t)ib - base] : vzero<VT>();
    for (int k = 1; k < st.ntaps; ++k) {
      ib = bc_index(bc, io + k, nx);
      if (ib < (uint64_t)nx) x0 = vadd(x0, x[(int64_t)ib - base]);
    }
    y = vfop(st.sub, st.c[0], x0, y);
  } else {
    const uint64_t ib = bc_index(bc, io, nx);
    if (ib < (uint64_t)nx) {
      const VT v = x[(int64_t)ib - base];
      y = st.sub ? vsub(y, v) : vadd(y, v);
    }
  }
  return y;
}

// ip_safe of the line kernel (taps from x-index j, dropped outside [0, nx)).
template <typename T, typename VT>
__device__ __forceinline__ VT ip_safe(const DevStep<T>& st, VT y, const VT* x, int64_t base,
                                      int64_t j, int64_t nx) {
  if (st.kind == K_GEN) {
    for (int k = 0; k < st.ntaps; ++k) {
      const int64_t ii = j + k;
      if (ii >= 0 && ii < nx) y = vfop(st.sub, st.c[k], x[ii - base], y);
    }
  } else {  // repeat
    VT x0 = (j >= 0 && j < nx) ? x[j - base] : vzero<VT>();
    for (int k = 1; k < st.ntaps; ++k) {
      const int64_t ii = j + k;
      if (ii >= 0 && ii < nx) x0 = vadd(x0, x[ii - base]);
    }
    y = vfop(st.sub, st.c[0], x0, y);
  }
  return y;
}

// Front fold of the line kernel (fold_front) on a band of nb elements.
template <typename T, typename VT>
__device__ __forceinline__ void fold_front(const DevStep<T>& st, int bc, VT* y, const VT* x,
                                           int64_t base, int64_t nb) {
  if (st.kind == K_UNIT) {
    for (int64_t i = st.fold_off, j = 0; i < 0 && j < nb; ++i, ++j) {
      const uint64_t io = bc_index(bc, i, nb);
      if (io < (uint64_t)nb && (int64_t)io != i) {
        VT& t = y[(int64_t)io - base];
        t = st.sub ? vsub(t, x[j - base]) : vadd(t, x[j - base]);
      }
    }
  } else {
    for (int64_t i = st.fold_off, j = 1 - st.ntaps; i < 0; ++i, ++j) {
      const uint64_t io = bc_index(bc, i, nb);
      if (io < (uint64_t)nb && (int64_t)io != i) {
        VT& t = y[(int64_t)io - base];
        t = ip_safe(st, t, x, base, j, nb);
      }
    }
  }
}

// Back fold of the line kernel (fold_back): every target (sel 0), or only
// the targets at or past n2 (sel 1) or before it (sel 2).
template <typename T, typename VT>
__device__ __forceinline__ void fold_back(const DevStep<T>& st, int bc, VT* y, const VT* x,
                                          int64_t base, int64_t nb, int64_t n2, int sel) {
  for (int64_t i = nb, j = nb + st.off; i < nb - st.off; ++i, ++j) {
    const uint64_t io = bc_index(bc, i, nb);
    if (io >= (uint64_t)nb || (int64_t)io == i) continue;
    if (sel != 0 && (sel == 1) != ((int64_t)io >= n2)) continue;
    VT& t = y[(int64_t)io - base];
    if (st.kind == K_UNIT) {
      if (j >= 0 && j < nb) t = st.sub ? vsub(t, x[j - base]) : vadd(t, x[j - base]);
    } else {
      t = ip_safe(st, t, x, base, j, nb);
    }
  }
}

// One edge's work for one step, before (post = false) or after the Zero
// update: windows y, x of band elements [base, base + E); sv keeps, for a
// normal step, the old values of the elements it recomputes (front: [0, nl);
// back: [nb - nr, nb)).  Out of line: one copy per lane type serves every
// step of every kernel.
template <typename T, typename VT>
__device__ __noinline__ void run(const DevStep<T>& st, const DevProgram<T>& prog, int bc,
                                 bool post, bool back, VT* y, const VT* x, VT* sv, int64_t base,
                                 int64_t nb, int nl, int nr) {
  const int64_t n2 = nb > st.nb ? nb - st.nb : 0;
  if (prog.normal) {
    if (!back) {
      for (int t = 0; t < nl; ++t) {
        if (!post) sv[t] = y[t - base];
        else y[t - base] = ip_bc(st, bc, sv[t], x, base, nb, t);
      }
    } else {
      for (int t = 0; t < nr; ++t) {
        const int64_t i = nb - nr + t;
        if (!post) sv[t] = y[i - base];
        else y[i - base] = ip_bc(st, bc, sv[t], x, base, nb, i);
      }
    }
    return;
  }
  if (!post) {
    if (!back) fold_front(st, bc, y, x, base, nb);
    else if (prog.across) fold_back(st, bc, y, x, base, nb, n2, 1);
  } else if (back) {
    fold_back(st, bc, y, x, base, nb, n2, prog.across ? 2 : 0);
  }
}

// The chunk side: copies the window of E pairs at the band end out of the
// register arrays (y, x of P pairs; the chunk holds band pairs
// [gp0, gp0 + P)), runs the edge work and copies y's window back.
template <int P, int E, bool BACK, typename T, typename VT, int PA>
__device__ __forceinline__ void call(const DevStep<T>& st, const DevProgram<T>& prog, int bc,
                                     bool post, VT (&y)[PA], const VT (&x)[PA], VT* sv,
                                     int64_t gp0, int64_t nb, int nl, int nr) {
  constexpr int LO = BACK ? P - E : 0;
  VT wy[E], wx[E];
#pragma unroll
  for (int t = 0; t < E; ++t) {
    wy[t] = y[LO + t];
    wx[t] = x[LO + t];
  }
  run<T, VT>(st, prog, bc, post, BACK, wy, wx, sv, gp0 + LO, nb, nl, nr);
#pragma unroll
  for (int t = 0; t < E; ++t) y[LO + t] = wy[t];
}

}  // namespace edge
}  // namespace lw
