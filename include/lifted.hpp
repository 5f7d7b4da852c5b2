// Drop-in C++ API: the four lifted::lwt overloads with the reference's
// exact signatures and default argument (src/lifted.hpp:13-39), backed by
// the B200 kernels through the C ABI in lifted_capi.h.
//
// Behaviour, as in the reference: the call returns when data_out holds the
// result; shapes and strides are in elements (strides may be negative);
// data_in == data_out is allowed.  Pointers may be host memory (staged
// through the GPU) or device memory (run on the legacy default stream, then
// synchronised).  Errors throw: std::invalid_argument for invalid arguments
// and for inputs on which the reference itself hangs or indexes out of
// bounds, std::bad_alloc for out-of-memory, std::runtime_error otherwise.
// n_threads is accepted and ignored (the CUDA grid replaces the thread
// pool).
#ifndef LIFTED_H_
#define LIFTED_H_

#if !(__cplusplus >= 202002L || _MSVC_LANG + 0L >= 202002L)
#error This file requires at least C++20 support.
#endif

#include "lifted-common.hpp"
#include "lifted-export.hpp"

namespace lifted {

LIFTED_DLLEXPORT void lwt(const Wavelet wvlt, const Transform op,
                          const BoundaryCondition bc, const size_v& shape,
                          const stride_v& stride_in,
                          const stride_v& stride_out, const size_v& axes,
                          const size_t levels, const float* data_in,
                          float* data_out, const size_t n_threads = 1);

LIFTED_DLLEXPORT void lwt(const Wavelet wvlt, const Transform op,
                          const BoundaryCondition bc, const size_v& shape,
                          const stride_v& stride_in,
                          const stride_v& stride_out, const size_v& axes,
                          const size_t levels, const double* data_in,
                          double* data_out, const size_t n_threads = 1);

LIFTED_DLLEXPORT void lwt(const Wavelet wvlt, const Transform op,
                          const BoundaryCondition bc, const size_v& shape,
                          const stride_v& stride_in,
                          const stride_v& stride_out, const size_v& axes,
                          const size_v& levels, const float* data_in,
                          float* data_out, const size_t n_threads = 1);

LIFTED_DLLEXPORT void lwt(const Wavelet wvlt, const Transform op,
                          const BoundaryCondition bc, const size_v& shape,
                          const stride_v& stride_in,
                          const stride_v& stride_out, const size_v& axes,
                          const size_v& levels, const double* data_in,
                          double* data_out, const size_t n_threads = 1);

}  // namespace lifted

#endif  // LIFTED_H_
