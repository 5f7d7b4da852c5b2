// Launch interface of the TMA-staged strided kernel (lw_col.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace lw {

struct ColParams;
using ColFn = cudaError_t (*)(const ColParams&, int, size_t, cudaStream_t);

// Launcher for (catalogue wavelet, transform, lines per lane); nullptr if
// not compiled.
ColFn pick_col(int wi, int op, int v);
// Dynamic shared memory of one CTA: staging buffer, mailbox, mbarrier.
size_t col_smem_bytes(int hmax, int v);

}  // namespace lw
