// Batched nD transforms of images with differing shapes, wavelets and level
// counts (C ABI lifted_lwt_batch_nd_f32/f64).
//
// The reference transforms one array per call (lifted::lwt,
// src/lifted.hpp:13-39); a training batch of images of different shapes is a
// loop of such calls.  Each image here is a dense C-order array transformed
// separably over all of its axes, exactly as
//     lifted_lwt_sep_xxx(wavelet, op, bc, ndim, shape, dense strides,
//                        ndim, {0, .., ndim-1}, levels, in + in_offset,
//                        out + out_offset, stream)
// would transform it.  Two ways to run a batch:
//   persistent  one launch of the batch engine for the whole batch: every
//               (image, axis) pass is cut into line items on the device
//               queue, and an image's later axes wait on its earlier ones
//               through completion counters (lw_batch_host.cpp,
//               run_batch_nd); images of every shape share the launch;
//   grouped     consecutive table entries with the same wavelet, shape and
//               levels, packed back to back in both buffers, form one group
//               that runs as one separable call over a (group, shape...)
//               view on the fast per-axis kernels: a few launches per axis
//               and group.
// The "batch_nd_mode" option picks one (0: automatic, the persistent launch
// once the batch has more than kGroupedMax groups; 1: persistent; 2:
// grouped).  Both are stream-ordered and can be captured into a CUDA graph
// (the persistent plan is built and cached on the first call outside a
// capture; a capture that meets an uncached batch runs it grouped).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "lifted_capi.h"
#include "lw_host.hpp"

namespace lw {
namespace {

// Largest number of groups the automatic mode still runs grouped.
constexpr size_t kGroupedMax = 4;

uint64_t numel_of(const lifted_image_t& im) {
  uint64_t n = 1;
  for (uint32_t d = 0; d < im.ndim; ++d) n *= im.shape[d];
  return n;
}

bool same_kind(const lifted_image_t& a, const lifted_image_t& b) {
  if (a.wavelet != b.wavelet || a.ndim != b.ndim) return false;
  for (uint32_t d = 0; d < a.ndim; ++d)
    if (a.shape[d] != b.shape[d] || a.levels[d] != b.levels[d]) return false;
  return true;
}

struct Span {
  uint64_t lo, hi;  // element range [lo, hi)
  size_t img;
};

template <typename T>
int batch_nd(uint32_t op, uint32_t bc, size_t nimg, const lifted_image_t* ims, const T* in,
             T* out, void* stream) {
  clear_error();
  if (nimg == 0) return LIFTED_OK;
  if (!ims || !in || !out) return set_error(LIFTED_EINVAL, "null pointer");
  if (!device_pointer(in) || !device_pointer(out))
    return set_error(LIFTED_EINVAL, "in and out must be device pointers");
  std::vector<Span> outs;
  outs.reserve(nimg);
  for (size_t i = 0; i < nimg; ++i) {
    const lifted_image_t& im = ims[i];
    if (im.ndim < 1 || im.ndim > 4)
      return set_error(LIFTED_EINVAL, "image %zu: ndim %u outside 1..4", i, im.ndim);
    uint64_t n = 1;
    for (uint32_t d = 0; d < im.ndim; ++d) {
      if (im.shape[d] == 0) return set_error(LIFTED_EINVAL, "image %zu: empty axis %u", i, d);
      if (n > (UINT64_MAX >> 1) / im.shape[d])
        return set_error(LIFTED_EINVAL, "image %zu: size overflow", i);
      n *= im.shape[d];
    }
    outs.push_back({im.out_offset, im.out_offset + n, i});
  }
  // outputs disjoint; no image's output may overlap another image's input
  // (the groups run in table order, not all at once)
  std::sort(outs.begin(), outs.end(), [](const Span& a, const Span& b) { return a.lo < b.lo; });
  for (size_t k = 1; k < outs.size(); ++k)
    if (outs[k].lo < outs[k - 1].hi)
      return set_error(LIFTED_EINVAL, "images %zu and %zu have overlapping outputs",
                       outs[k - 1].img, outs[k].img);
  const char* ib = (const char*)in;
  const char* ob = (const char*)out;
  for (size_t i = 0; i < nimg; ++i) {
    const lifted_image_t& im = ims[i];
    const char* lo = ib + im.in_offset * sizeof(T);
    const char* hi = lo + numel_of(im) * sizeof(T);
    // output spans that intersect [lo, hi), found by binary search
    auto it = std::upper_bound(outs.begin(), outs.end(), lo, [&](const char* v, const Span& s) {
      return v < ob + s.hi * sizeof(T);
    });
    for (; it != outs.end() && ob + it->lo * sizeof(T) < hi; ++it)
      if (it->img != i)
        return set_error(LIFTED_EINVAL, "image %zu's input overlaps image %zu's output", i,
                         it->img);
  }
  // groups of consecutive, identically shaped, packed images
  size_t ngroups = 0;
  for (size_t i = 0; i < nimg;) {
    const uint64_t n = numel_of(ims[i]);
    size_t j = i + 1;
    while (j < nimg && same_kind(ims[i], ims[j]) &&
           ims[j].in_offset == ims[j - 1].in_offset + n &&
           ims[j].out_offset == ims[j - 1].out_offset + n)
      ++j;
    ++ngroups;
    i = j;
  }
  const int mode = batch_nd_mode();
  bool persistent = mode == 1 || (mode == 0 && ngroups > kGroupedMax);
  // line items run an image in place only when its input and output spans
  // coincide or are disjoint
  for (size_t k = 0; k < nimg && persistent; ++k) {
    const char* lo = ib + ims[k].in_offset * sizeof(T);
    const char* o = ob + ims[k].out_offset * sizeof(T);
    const size_t bytes = numel_of(ims[k]) * sizeof(T);
    if (lo != o && lo < o + bytes && o < lo + bytes) persistent = false;
  }
  if (persistent) {
    bool ran = false;
    const int rc = run_batch_nd<T>(op, bc, nimg, ims, in, out, (cudaStream_t)stream, &ran);
    if (rc != LIFTED_OK || ran) return rc;
  }
  size_t i = 0;
  while (i < nimg) {
    const lifted_image_t& a = ims[i];
    const uint64_t n = numel_of(a);
    size_t j = i + 1;
    while (j < nimg && same_kind(a, ims[j]) && ims[j].in_offset == ims[j - 1].in_offset + n &&
           ims[j].out_offset == ims[j - 1].out_offset + n)
      ++j;
    const size_t g = j - i;
    size_t shape[5], axes[4], levels[4];
    ptrdiff_t stride[5];
    const size_t nd = a.ndim + (g > 1 ? 1 : 0);
    size_t k = 0;
    if (g > 1) shape[k++] = g;
    for (uint32_t d = 0; d < a.ndim; ++d) {
      shape[k++] = (size_t)a.shape[d];
      axes[d] = (g > 1 ? 1 : 0) + d;
      levels[d] = a.levels[d];
    }
    ptrdiff_t s = 1;
    for (size_t d = nd; d-- > 0;) {
      stride[d] = s;
      s *= (ptrdiff_t)shape[d];
    }
    int rc;
    if constexpr (sizeof(T) == 4)
      rc = lifted_lwt_sep_f32(a.wavelet, op, bc, nd, shape, stride, stride, a.ndim, axes, levels,
                              in + a.in_offset, out + a.out_offset, stream);
    else
      rc = lifted_lwt_sep_f64(a.wavelet, op, bc, nd, shape, stride, stride, a.ndim, axes, levels,
                              in + a.in_offset, out + a.out_offset, stream);
    if (rc != LIFTED_OK) return rc;  // the error names the failing call
    i = j;
  }
  return LIFTED_OK;
}

}  // namespace
}  // namespace lw

extern "C" {

LIFTED_CAPI int lifted_lwt_batch_nd_f32(uint32_t op, uint32_t bc, size_t nimages,
                                        const lifted_image_t* images, const float* in,
                                        float* out, void* stream) {
  return lw::batch_nd<float>(op, bc, nimages, images, in, out, stream);
}
LIFTED_CAPI int lifted_lwt_batch_nd_f64(uint32_t op, uint32_t bc, size_t nimages,
                                        const lifted_image_t* images, const double* in,
                                        double* out, void* stream) {
  return lw::batch_nd<double>(op, bc, nimages, images, in, out, stream);
}

}  // extern "C"
