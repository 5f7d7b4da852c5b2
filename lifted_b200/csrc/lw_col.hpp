// Launch interface of the TMA-staged strided kernel (lw_col.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace lw {

template <typename T>
struct ColParams;
template <typename T>
using ColFn = cudaError_t (*)(const ColParams<T>&, int, size_t, cudaStream_t);

// Launcher for (catalogue wavelet, transform, lines per lane, lines whose
// length is not a multiple of 32); nullptr if not compiled.  float64, and
// such lines, have one line per lane only.
// edge: the instantiation with exact band edges for the Constant, Symmetric
// and Reflect boundaries (compiled wavelets, whole chunks).
ColFn<float> pick_col_f32(int wi, int op, int v, bool em, bool edge);
ColFn<double> pick_col_f64(int wi, int op, bool em, bool edge);
// The plain-load instantiations (staging without TMA, for strides, line
// counts or bases that are not multiples of 16 bytes; Zero boundary, one
// line per lane, any line length); nullptr if not compiled.
ColFn<float> pick_col_ldg_f32(int wi, int op);
ColFn<double> pick_col_ldg_f64(int wi, int op);
// Dynamic shared memory of one CTA: staging buffer, mailbox (mb_bufs
// buffers), mbarrier.
size_t col_smem_bytes(int hmax, int v, int elem_bytes, int mb_bufs);

}  // namespace lw
