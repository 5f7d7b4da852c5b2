// C entry points over the reference implementation, for use as a checker.
//
// Test infrastructure only: oracle/build_ref.sh compiles this file together
// with the reference's own, unmodified sources (src/lifted-*.cpp of
// jcapriot/lifted) against the Highway stand-in in oracle/hwy_shim into
// oracle/_ref/liblifted_ref_<variant>.so.  Only tests/, the smoke check and
// bench.py's CPU baseline load that library.  Nothing here is part of the GPU
// product.
//
// Exported:
//   ref_lwt_sep_{f32,f64}  -> lifted::lwt(..., const size_v& levels, ...)
//                            (src/lifted.hpp:27-39)
//   ref_lwt_{f32,f64}      -> lifted::lwt(..., const size_t level, ...)
//                            (src/lifted.hpp:13-25)
//   ref_fixed_apply_f64/f32 -> FixedTransform<W>::apply on pre-split s/d
//                            buffers (src/lifted-drivers-inl.hpp:37-64), the
//                            step-level contract that tests/test_single_levels
//                            .cpp:47-51 exercises; W is a catalogue wavelet
//                            (kind 0) or one of the 25 mock step programs of
//                            tests/test_helpers.h:102-356 (kind 1).
//   ref_lanes_{f32,f64}, ref_wavelet_width, ref_max_level
// Every call returns 0 on success, 1 on std::invalid_argument, 2 on any
// other exception.
#include <cstdint>
#include <cstring>
#include <exception>
#include <functional>
#include <stdexcept>
#include <vector>

#include "hwy/highway.h"
#include "lifted.hpp"
#include "lifted-inl.hpp"

namespace {

using lifted::size_v;
using lifted::stride_v;

template <typename Fn>
int guarded(Fn&& fn) {
  try {
    fn();
    return 0;
  } catch (const std::invalid_argument&) {
    return 1;
  } catch (...) {
    return 2;
  }
}

template <typename T>
int sep_call(uint32_t w, uint32_t op, uint32_t bc, size_t ndim,
             const size_t* shape, const ptrdiff_t* sin, const ptrdiff_t* sout,
             size_t naxes, const size_t* axes, const size_t* levels,
             const T* in, T* out, size_t nthreads) {
  return guarded([&] {
    size_v shp(shape, shape + ndim);
    stride_v si(sin, sin + ndim), so(sout, sout + ndim);
    size_v ax(axes, axes + naxes), lv(levels, levels + naxes);
    lifted::lwt(lifted::Wavelet(w), lifted::Transform(op),
                lifted::BoundaryCondition(bc), shp, si, so, ax, lv, in, out,
                nthreads);
  });
}

template <typename T>
int nonsep_call(uint32_t w, uint32_t op, uint32_t bc, size_t ndim,
                const size_t* shape, const ptrdiff_t* sin,
                const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                size_t level, const T* in, T* out, size_t nthreads) {
  return guarded([&] {
    size_v shp(shape, shape + ndim);
    stride_v si(sin, sin + ndim), so(sout, sout + ndim);
    size_v ax(axes, axes + naxes);
    lifted::lwt(lifted::Wavelet(w), lifted::Transform(op),
                lifted::BoundaryCondition(bc), shp, si, so, ax, level, in,
                out, nthreads);
  });
}

}  // namespace

// ---------------------------------------------------------------------------
// Mock step programs.  These restate the 25 single-step test programs that
// the reference's step-level suite is parameterised over, in the same order
// (index = MockWavelet value).
namespace lifted {
namespace detail {
namespace oracle_mocks {
using UO = UpdateOperation;
#define ORACLE_MOCK(NAME, ...)                                   \
  template <typename T>                                          \
  struct NAME {                                                  \
    using type = T;                                              \
    constexpr static auto steps = std::make_tuple(__VA_ARGS__);  \
  };
ORACLE_MOCK(M0, update_s<T>(0, 1.2))
ORACLE_MOCK(M1, update_s<T>(-5, 1.2, 1.5, 1.6))
ORACLE_MOCK(M2, update_s<T>(3, 1.2, 1.5, 1.6))
ORACLE_MOCK(M3, update_s<T>(-2, 1.2, 1.3, 1.5, -1.2, -3.2))
ORACLE_MOCK(M4, update_d<T>(0, 0.5))
ORACLE_MOCK(M5, update_d<T>(-5, 1.2, 1.5, 1.6))
ORACLE_MOCK(M6, update_d<T>(3, 1.2, 1.5, 1.6))
ORACLE_MOCK(M7, update_d<T>(-2, 0.5, 1.203, 4.2, 33.213))
ORACLE_MOCK(M8, unit_update_s<T, UO::add>(0))
ORACLE_MOCK(M9, unit_update_s<T, UO::sub>(3))
ORACLE_MOCK(M10, unit_update_s<T, UO::add>(-3))
ORACLE_MOCK(M11, unit_update_d<T, UO::sub>(0))
ORACLE_MOCK(M12, unit_update_d<T, UO::add>(3))
ORACLE_MOCK(M13, unit_update_d<T, UO::sub>(-3))
ORACLE_MOCK(M14, (repeat_update_s<T, 1>(0, 0.5)))
ORACLE_MOCK(M15, (repeat_update_s<T, 3>(-4, 0.5)))
ORACLE_MOCK(M16, (repeat_update_s<T, 3>(2, 0.5)))
ORACLE_MOCK(M17, (repeat_update_s<T, 3>(-1, 0.5)))
ORACLE_MOCK(M18, (repeat_update_d<T, 1>(0, 0.5)))
ORACLE_MOCK(M19, (repeat_update_d<T, 3>(-4, 0.5)))
ORACLE_MOCK(M20, (repeat_update_d<T, 3>(2, 0.5)))
ORACLE_MOCK(M21, (repeat_update_d<T, 3>(-1, 0.5)))
ORACLE_MOCK(M22, ScaleStep<T>(0.124))
ORACLE_MOCK(M23, ScaleStep<T>(5.23, 0.124))
ORACLE_MOCK(M24, update_s<T>(-5, 1.2, 1.3, 1.5, -1.2, -3.2),
            update_d<T>(-5, 0.5, 1.203, 4.2, 33.213), ScaleStep<T>(0.124))
#undef ORACLE_MOCK
}  // namespace oracle_mocks
}  // namespace detail
}  // namespace lifted

namespace {
namespace dh = lifted::detail::HWY_NAMESPACE;
namespace om = lifted::detail::oracle_mocks;
using lifted::BoundaryCondition;
using lifted::Transform;

template <template <typename> class W, typename T>
void apply_one(uint32_t op, uint32_t dir, BoundaryCondition bc, T* s, T* d,
               size_t ns, size_t nd) {
  using FT = dh::FixedTransform<W<T>>;
  namespace ld = lifted::detail;
  auto go = [&](auto tf) {
    if (dir == 0)
      FT::apply(tf, ld::Along(), bc, s, d, ns, nd);
    else
      FT::apply(tf, ld::Across(), bc, s, d, ns, nd);
  };
  switch (op) {
    case 0: go(ld::Forward()); break;
    case 1: go(ld::Inverse()); break;
    case 2: go(ld::ForwardAdjoint()); break;
    case 3: go(ld::InverseAdjoint()); break;
    default: throw std::invalid_argument("bad transform");
  }
}

template <typename T>
void apply_mock(uint32_t idx, uint32_t op, uint32_t dir, BoundaryCondition bc,
                T* s, T* d, size_t ns, size_t nd) {
  switch (idx) {
#define M(I) \
  case I: apply_one<om::M##I, T>(op, dir, bc, s, d, ns, nd); return;
    M(0) M(1) M(2) M(3) M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12)
    M(13) M(14) M(15) M(16) M(17) M(18) M(19) M(20) M(21) M(22) M(23) M(24)
#undef M
    default: throw std::invalid_argument("bad mock index");
  }
}

template <typename T>
void apply_catalogue(uint32_t w, uint32_t op, uint32_t dir,
                     BoundaryCondition bc, T* s, T* d, size_t ns, size_t nd) {
  switch (lifted::Wavelet(w)) {
#define X(name, val)                                                  \
  case lifted::Wavelet::name:                                         \
    apply_one<lifted::name, T>(op, dir, bc, s, d, ns, nd);            \
    return;
    LIFTED_WAVELETS
#undef X
    default: throw std::invalid_argument("bad wavelet");
  }
}

}  // namespace

extern "C" {

int ref_lwt_sep_f32(uint32_t w, uint32_t op, uint32_t bc, size_t ndim,
                    const size_t* shape, const ptrdiff_t* sin,
                    const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                    const size_t* levels, const float* in, float* out,
                    size_t nthreads) {
  return sep_call<float>(w, op, bc, ndim, shape, sin, sout, naxes, axes,
                         levels, in, out, nthreads);
}

int ref_lwt_sep_f64(uint32_t w, uint32_t op, uint32_t bc, size_t ndim,
                    const size_t* shape, const ptrdiff_t* sin,
                    const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                    const size_t* levels, const double* in, double* out,
                    size_t nthreads) {
  return sep_call<double>(w, op, bc, ndim, shape, sin, sout, naxes, axes,
                          levels, in, out, nthreads);
}

int ref_lwt_f32(uint32_t w, uint32_t op, uint32_t bc, size_t ndim,
                const size_t* shape, const ptrdiff_t* sin,
                const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                size_t level, const float* in, float* out, size_t nthreads) {
  return nonsep_call<float>(w, op, bc, ndim, shape, sin, sout, naxes, axes,
                            level, in, out, nthreads);
}

int ref_lwt_f64(uint32_t w, uint32_t op, uint32_t bc, size_t ndim,
                const size_t* shape, const ptrdiff_t* sin,
                const ptrdiff_t* sout, size_t naxes, const size_t* axes,
                size_t level, const double* in, double* out,
                size_t nthreads) {
  return nonsep_call<double>(w, op, bc, ndim, shape, sin, sout, naxes, axes,
                             level, in, out, nthreads);
}

// kind 0: catalogue wavelet (value = Wavelet enum); kind 1: mock index 0..24.
// dir 0: Along (s/d contiguous), 1: Across (s/d hold `lanes` interleaved
// lines, element i of line j at [i * lanes + j]).
int ref_fixed_apply_f64(uint32_t kind, uint32_t w, uint32_t op, uint32_t dir,
                        uint32_t bc, double* s, double* d, size_t ns,
                        size_t nd) {
  return guarded([&] {
    if (kind == 0)
      apply_catalogue<double>(w, op, dir, BoundaryCondition(bc), s, d, ns, nd);
    else
      apply_mock<double>(w, op, dir, BoundaryCondition(bc), s, d, ns, nd);
  });
}

int ref_fixed_apply_f32(uint32_t kind, uint32_t w, uint32_t op, uint32_t dir,
                        uint32_t bc, float* s, float* d, size_t ns,
                        size_t nd) {
  return guarded([&] {
    if (kind == 0)
      apply_catalogue<float>(w, op, dir, BoundaryCondition(bc), s, d, ns, nd);
    else
      apply_mock<float>(w, op, dir, BoundaryCondition(bc), s, d, ns, nd);
  });
}

size_t ref_lanes_f32(void) { return hwy::N_SHIM::Lanes(hwy::N_SHIM::ScalableTag<float>()); }
size_t ref_lanes_f64(void) { return hwy::N_SHIM::Lanes(hwy::N_SHIM::ScalableTag<double>()); }

// Returns (size_t)-1 for an unknown wavelet value.
size_t ref_wavelet_width(uint32_t w) {
  switch (lifted::Wavelet(w)) {
#define X(name, val) \
  case lifted::Wavelet::name: return lifted::name<double>::width;
    LIFTED_WAVELETS
#undef X
    default: return (size_t)-1;
  }
}

// The reference's max_level(width, n) (src/lifted-common.hpp:1099-1108).
// Never call it with width == 1: the reference loops forever there.
size_t ref_max_level(size_t width, size_t n) {
  return lifted::max_level(width, n);
}

}  // extern "C"
