// Batched uneven-length 1D transforms: work items of the persistent batch
// kernel (lw_batch_kernel.cuh) and its launch interface.
//
// A batch is many contiguous 1D signals, each with its own length, catalogue
// wavelet and level count; each is transformed exactly as the separable
// driver transforms a one-dimensional array (src/lifted-drivers-inl.hpp:
// 417-486 with one axis).  The host planner cuts every signal into work
// items; one persistent launch pulls the items from a device queue in order.
//
//   whole item   the signal's band of level lev0 fits in shared memory: the
//                remaining levels run on it with the exact general step code
//                (every boundary condition);
//   tile item    a long band (Zero boundary only): a window
//                [t0 - halo, t1 + halo) of the band runs `nlev` levels in
//                shared memory and stores only the interior [t0, t1) of every
//                detail band and of the last approximation band.  The halo
//                covers the values a window edge corrupts over those levels,
//                so interior results are those of the whole band.
//
// Forward-stepping transforms (Forward, InverseAdjoint) go fine to coarse:
// level-group tiles first, a whole item for the coarsest levels last.
// Reverse-stepping transforms (Inverse, ForwardAdjoint) go coarse to fine.
// An item whose input band another item produces waits (bounded) on that
// producer group's completion counter; the queue order puts every producer
// before its consumers, so waits always end.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "lw_types.hpp"

namespace lw {

enum BatchItemKind : int32_t {
  BI_WHOLE_FWD = 0,
  BI_WHOLE_REV = 1,
  BI_TILE_FWD = 2,
  BI_TILE_REV = 3,
  BI_LINES_FWD = 4,  // line items of an nD image's axis pass (below)
  BI_LINES_REV = 5
};

// Lines of one axis pass of a dense C-order nD image (line items of a
// batch of nD images): the lines along the axis, enumerated over the other
// dims fastest first, so consecutive line indices of a strided axis are
// adjacent in memory.  Element i of line L sits at
// base(L) + i * sa, base(L) = sum over the other dims of idx_d * ostride_d.
struct BatchAxisGeom {
  int64_t n;           // line length
  int64_t sa;          // element stride along the axis
  int64_t oshape[3];   // other dims, fastest first (1 where absent)
  int64_t ostride[3];
};
// Where a band lives.
enum BandSel : int32_t { BS_IN = 0, BS_OUT = 1, BS_SCRATCH = 2 };

struct BatchItem {
  int32_t kind;
  int32_t prog;         // index into the program table
  int32_t sig;          // signal index (diagnostics)
  int32_t lev0;         // level of the finest band the item touches
  int32_t nlev;         // levels the item runs
  int32_t src_sel;      // forward: band lev0; reverse: approximation lev0+nlev
  int32_t dst_sel;      // forward: approximation lev0+nlev; reverse: band lev0
  int32_t wait_ctr;     // completion counter to wait for (-1: none)
  int32_t wait_target;  // value that counter must reach
  int32_t done_ctr;     // counter this item increments when done (-1: none)
  int32_t geo;          // line items: index of the axis pass's geometry
  int32_t zfast;        // whole and line items: 1 = Zero boundary, direct
                        // step code (zero_step), the host having checked
                        // that no level's edge ranges overlap
  int64_t n0;           // signal length (line items: line length)
  int64_t in_off;       // signal offset in `in` (elements)
  int64_t out_off;      // signal offset in `out`
  int64_t src_off;      // offset of the source band in its array
  int64_t dst_off;      // offset of the destination band in its array
  int64_t t0, t1;       // tile interior, samples of band lev0 (line
                        // items: the lines [t0, t1) of the pass)
  int64_t halo;         // tile halo per side, samples of band lev0
  int64_t gbuf;         // whole item over global buffers: scratch offset of
                        // its 1.5 * band elements (-1: shared memory; line
                        // items: -2 = the CTA's own slot of global scratch)
};

template <typename T>
struct BatchParams {
  const T* in;
  T* out;
  T* scratch;
  const BatchItem* items;
  const DevProgram<T>* progs;
  int32_t* head;       // dequeue counter, zero at launch
  int32_t* counters;   // completion counters, zero at launch
  int32_t* error;      // first item whose wait gave up, plus one (0: none)
  int32_t nitems;
  int32_t bc;
  int64_t buf_elems;   // shared-memory band capacity (elements, 1.5x band)
  int32_t spin_limit;  // polls of a completion counter before giving up
  int32_t pad_;
  const BatchAxisGeom* geos;  // line items: axis pass geometries
  int64_t slot_off;    // line items longer than shared memory: CTA b works
  int64_t slot_elems;  //   in scratch[slot_off + b * slot_elems, ...)
};

// Shared memory of the batch kernel for a band capacity of `buf_elems`.
template <typename T>
constexpr size_t batch_smem_bytes(int64_t buf_elems) {
  return ((sizeof(DevProgram<T>) + 15) / 16) * 16 + (size_t)buf_elems * sizeof(T);
}

cudaError_t launch_batch(const BatchParams<float>& p, int grid, int block,
                         size_t smem, cudaStream_t stream);
cudaError_t launch_batch(const BatchParams<double>& p, int grid, int block,
                         size_t smem, cudaStream_t stream);
// Resident CTAs per SM of the batch kernel at this block and shared memory.
int batch_occupancy(int dtype_bytes, int block, size_t smem);

}  // namespace lw
