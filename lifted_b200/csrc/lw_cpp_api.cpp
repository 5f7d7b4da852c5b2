// The drop-in C++ overloads of lifted::lwt (include/lifted.hpp) over the C
// ABI.  Replaces src/lifted-float.cpp:20-30, src/lifted-double.cpp:20-30,
// src/lifted-sep-float.cpp:20-30 and src/lifted-sep-double.cpp:20-30.
#define LIFTED_SHARED_DEFINE 1
#define LIFTED_EXPORTS 1
#include <cuda_runtime.h>

#include <new>
#include <stdexcept>
#include <string>

#include "../../include/lifted.hpp"
#include "../../include/lifted_capi.h"

namespace lifted {
namespace {

void raise_for(int rc) {
  if (rc == LIFTED_OK) return;
  std::string msg = std::string(lifted_status_string(rc)) + ": " +
                    lifted_last_error();
  switch (rc) {
    case LIFTED_EINVAL:
    case LIFTED_EDEGENERATE:
    case LIFTED_ETOOLARGE:
      throw std::invalid_argument(msg);
    case LIFTED_ENOMEM:
      throw std::bad_alloc();
    default:
      throw std::runtime_error(msg);
  }
}

void check_sizes(const size_v& shape, const stride_v& si, const stride_v& so) {
  if (si.size() != shape.size() || so.size() != shape.size())
    throw std::invalid_argument("stride vectors must match the shape's rank");
}

// Completes device-pointer calls before returning, like the reference.
void finish(int rc) {
  if (rc == LIFTED_OK) {
    cudaError_t e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("cudaStreamSynchronize: ") +
                               cudaGetErrorString(e));
  }
  raise_for(rc);
}

}  // namespace

void lwt(const Wavelet wvlt, const Transform op, const BoundaryCondition bc,
         const size_v& shape, const stride_v& stride_in,
         const stride_v& stride_out, const size_v& axes, const size_t levels,
         const float* data_in, float* data_out, const size_t) {
  check_sizes(shape, stride_in, stride_out);
  finish(lifted_lwt_f32((uint32_t)wvlt, (uint32_t)op, (uint32_t)bc,
                        shape.size(), shape.data(), stride_in.data(),
                        stride_out.data(), axes.size(), axes.data(), levels,
                        data_in, data_out, nullptr));
}

void lwt(const Wavelet wvlt, const Transform op, const BoundaryCondition bc,
         const size_v& shape, const stride_v& stride_in,
         const stride_v& stride_out, const size_v& axes, const size_t levels,
         const double* data_in, double* data_out, const size_t) {
  check_sizes(shape, stride_in, stride_out);
  finish(lifted_lwt_f64((uint32_t)wvlt, (uint32_t)op, (uint32_t)bc,
                        shape.size(), shape.data(), stride_in.data(),
                        stride_out.data(), axes.size(), axes.data(), levels,
                        data_in, data_out, nullptr));
}

void lwt(const Wavelet wvlt, const Transform op, const BoundaryCondition bc,
         const size_v& shape, const stride_v& stride_in,
         const stride_v& stride_out, const size_v& axes, const size_v& levels,
         const float* data_in, float* data_out, const size_t) {
  check_sizes(shape, stride_in, stride_out);
  if (levels.size() < axes.size())
    throw std::invalid_argument("levels must be the same length as axes");
  finish(lifted_lwt_sep_f32((uint32_t)wvlt, (uint32_t)op, (uint32_t)bc,
                            shape.size(), shape.data(), stride_in.data(),
                            stride_out.data(), axes.size(), axes.data(),
                            levels.data(), data_in, data_out, nullptr));
}

void lwt(const Wavelet wvlt, const Transform op, const BoundaryCondition bc,
         const size_v& shape, const stride_v& stride_in,
         const stride_v& stride_out, const size_v& axes, const size_v& levels,
         const double* data_in, double* data_out, const size_t) {
  check_sizes(shape, stride_in, stride_out);
  if (levels.size() < axes.size())
    throw std::invalid_argument("levels must be the same length as axes");
  finish(lifted_lwt_sep_f64((uint32_t)wvlt, (uint32_t)op, (uint32_t)bc,
                            shape.size(), shape.data(), stride_in.data(),
                            stride_out.data(), axes.size(), axes.data(),
                            levels.data(), data_in, data_out, nullptr));
}

}  // namespace lifted
