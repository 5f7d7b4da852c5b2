// Minimal stand-in for the subset of Google Highway that the lifted
// reference sources use, so that those sources compile unchanged without
// Highway (which is neither vendored nor installed on this image).
//
// This file is test infrastructure for the oracle: it is only ever compiled
// together with the reference's own sources into oracle/_ref/ (see
// oracle/build_ref.sh) and is never part of the GPU library.
//
// It provides a single compile-time target.  The vector width in bytes is
// set by SHIM_VEC_BYTES (0 = scalar, one lane; 32 = AVX2-width; 64 =
// AVX-512-width).  Lane operations are written over GCC vector extensions.
// MulAdd / NegMulAdd are always fused (one rounding), which is what Highway
// does on every x86 target that has FMA.
//
// Ops provided (the complete list found by grep over the reference's src/):
//   ScalableTag, VFromD, Lanes, Set, Zero, Undefined, Load, LoadU, LoadN,
//   Store, StoreU, StoreN, Add, Sub, Mul, MulAdd, NegMulAdd,
//   LoadInterleaved2, StoreInterleaved2, hwy::AllocateAligned
// and the macros HWY_NAMESPACE, HWY_ATTR, HWY_INLINE, HWY_NOINLINE,
// HWY_RESTRICT, HWY_LANES_CONSTEXPR, HWY_HAVE_CONSTEXPR_LANES,
// HWY_BEFORE_NAMESPACE, HWY_AFTER_NAMESPACE, HWY_EXPORT,
// HWY_DYNAMIC_DISPATCH, HWY_ONCE.
#ifndef LIFTED_ORACLE_HWY_SHIM_H_
#define LIFTED_ORACLE_HWY_SHIM_H_

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>

#ifndef SHIM_VEC_BYTES
#define SHIM_VEC_BYTES 32
#endif

#define HWY_NAMESPACE N_SHIM
#define HWY_ATTR
#define HWY_INLINE inline __attribute__((always_inline))
#define HWY_NOINLINE __attribute__((noinline))
#define HWY_RESTRICT __restrict__
#define HWY_LANES_CONSTEXPR constexpr
#define HWY_HAVE_CONSTEXPR_LANES 1
#define HWY_BEFORE_NAMESPACE() static_assert(true, "hwy shim")
#define HWY_AFTER_NAMESPACE() static_assert(true, "hwy shim")
#define HWY_ONCE 1
#define HWY_EXPORT(FUNC) static_assert(true, "hwy shim export")
#define HWY_DYNAMIC_DISPATCH(FUNC) HWY_NAMESPACE::FUNC

namespace hwy {

struct ShimAlignedFree {
  void operator()(void* p) const noexcept { std::free(p); }
};

template <typename T>
using AlignedFreeUniquePtr = std::unique_ptr<T, ShimAlignedFree>;

// Highway returns 64-byte aligned, uninitialised storage.
template <typename T>
AlignedFreeUniquePtr<T[]> AllocateAligned(const size_t items) {
  size_t bytes = items * sizeof(T);
  bytes = (bytes + 63) / 64 * 64;
  if (bytes == 0) bytes = 64;
  void* p = std::aligned_alloc(64, bytes);
  if (!p) throw std::bad_alloc();
  return AlignedFreeUniquePtr<T[]>(static_cast<T*>(p));
}

namespace N_SHIM {

template <typename T, size_t N>
struct Simd {
  using T_ = T;
  static constexpr size_t kLanes = N;
  constexpr Simd() = default;
};

template <typename T>
using ScalableTag =
    Simd<T, (SHIM_VEC_BYTES == 0 ? 1 : SHIM_VEC_BYTES / sizeof(T))>;

template <typename T, size_t N>
struct Vec {
  typedef T raw_t __attribute__((vector_size(N * sizeof(T))));
  raw_t raw;
};

// One-lane vectors stay plain scalars: GCC vector extensions need a
// power-of-two size of at least one element, which holds, but a scalar keeps
// the lanes=1 build bit-identical to straight-line scalar code.
template <typename T>
struct Vec<T, 1> {
  T raw;
};

template <class D>
using VFromD = Vec<typename D::T_, D::kLanes>;

template <typename T, size_t N>
constexpr size_t Lanes(Simd<T, N>) {
  return N;
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> Set(Simd<T, N>, T value) {
  Vec<T, N> v;
  if constexpr (N == 1) {
    v.raw = value;
  } else {
    for (size_t i = 0; i < N; ++i) v.raw[i] = value;
  }
  return v;
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> Zero(Simd<T, N> d) {
  return Set(d, T(0));
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> Undefined(Simd<T, N> d) {
  return Set(d, T(0));
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> LoadU(Simd<T, N>, const T* HWY_RESTRICT p) {
  Vec<T, N> v;
  std::memcpy(&v.raw, p, N * sizeof(T));
  return v;
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> Load(Simd<T, N> d, const T* HWY_RESTRICT p) {
  return LoadU(d, p);
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> LoadN(Simd<T, N> d, const T* HWY_RESTRICT p,
                           size_t max_lanes) {
  Vec<T, N> v = Zero(d);
  const size_t n = max_lanes < N ? max_lanes : N;
  std::memcpy(&v.raw, p, n * sizeof(T));
  return v;
}

template <typename T, size_t N>
HWY_INLINE void StoreU(Vec<T, N> v, Simd<T, N>, T* HWY_RESTRICT p) {
  std::memcpy(p, &v.raw, N * sizeof(T));
}

template <typename T, size_t N>
HWY_INLINE void Store(Vec<T, N> v, Simd<T, N> d, T* HWY_RESTRICT p) {
  StoreU(v, d, p);
}

template <typename T, size_t N>
HWY_INLINE void StoreN(Vec<T, N> v, Simd<T, N>, T* HWY_RESTRICT p,
                       size_t max_lanes) {
  const size_t n = max_lanes < N ? max_lanes : N;
  std::memcpy(p, &v.raw, n * sizeof(T));
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> Add(Vec<T, N> a, Vec<T, N> b) {
  a.raw = a.raw + b.raw;
  return a;
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> Sub(Vec<T, N> a, Vec<T, N> b) {
  a.raw = a.raw - b.raw;
  return a;
}

template <typename T, size_t N>
HWY_INLINE Vec<T, N> Mul(Vec<T, N> a, Vec<T, N> b) {
  a.raw = a.raw * b.raw;
  return a;
}

// mul * x + add, one rounding.
template <typename T, size_t N>
HWY_INLINE Vec<T, N> MulAdd(Vec<T, N> mul, Vec<T, N> x, Vec<T, N> add) {
  Vec<T, N> r;
  if constexpr (N == 1) {
    r.raw = std::fma(mul.raw, x.raw, add.raw);
  } else {
    for (size_t i = 0; i < N; ++i)
      r.raw[i] = std::fma(mul.raw[i], x.raw[i], add.raw[i]);
  }
  return r;
}

// add - mul * x, one rounding.
template <typename T, size_t N>
HWY_INLINE Vec<T, N> NegMulAdd(Vec<T, N> mul, Vec<T, N> x, Vec<T, N> add) {
  Vec<T, N> r;
  if constexpr (N == 1) {
    r.raw = std::fma(-mul.raw, x.raw, add.raw);
  } else {
    for (size_t i = 0; i < N; ++i)
      r.raw[i] = std::fma(-mul.raw[i], x.raw[i], add.raw[i]);
  }
  return r;
}

template <typename T, size_t N>
HWY_INLINE void LoadInterleaved2(Simd<T, N>, const T* HWY_RESTRICT p,
                                 Vec<T, N>& v0, Vec<T, N>& v1) {
  if constexpr (N == 1) {
    v0.raw = p[0];
    v1.raw = p[1];
  } else {
    for (size_t i = 0; i < N; ++i) {
      v0.raw[i] = p[2 * i];
      v1.raw[i] = p[2 * i + 1];
    }
  }
}

template <typename T, size_t N>
HWY_INLINE void StoreInterleaved2(Vec<T, N> v0, Vec<T, N> v1, Simd<T, N>,
                                  T* HWY_RESTRICT p) {
  if constexpr (N == 1) {
    p[0] = v0.raw;
    p[1] = v1.raw;
  } else {
    for (size_t i = 0; i < N; ++i) {
      p[2 * i] = v0.raw[i];
      p[2 * i + 1] = v1.raw[i];
    }
  }
}

}  // namespace N_SHIM
}  // namespace hwy

#endif  // LIFTED_ORACLE_HWY_SHIM_H_
