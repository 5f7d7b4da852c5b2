// Lane arithmetic of the register kernels: a lane holds V adjacent lines
// (V = 2 packs two float32 lines into FP32x2 arithmetic), and every helper
// is the exact element-wise equivalent of the scalar form (IEEE round to
// nearest, no contraction beyond the explicit fused multiply-adds).
#pragma once

#include <cstdint>

#include "lw_line_kernel.cuh"

namespace lw {

// Lane value types: V adjacent lines per lane.  The arithmetic helpers are
// exact element-wise equivalents of the scalar forms (IEEE round to nearest;
// packed FP32x2 on sm_100 for float2).
template <typename T, int V>
struct LaneVec;
template <typename T>
struct LaneVec<T, 1> {
  using type = T;
};
template <>
struct LaneVec<float, 2> {
  using type = float2;
};
template <>
struct LaneVec<double, 2> {
  using type = double2;
};

__device__ __forceinline__ float vfop(int sub, float c, float x, float y) {
  return fop(sub, c, x, y);
}
__device__ __forceinline__ double vfop(int sub, double c, double x, double y) {
  return fop(sub, c, x, y);
}
__device__ __forceinline__ float2 vfop(int sub, float c, float2 x, float2 y) {
  const float cc = sub ? -c : c;
  return __ffma2_rn(make_float2(cc, cc), x, y);
}
__device__ __forceinline__ double2 vfop(int sub, double c, double2 x, double2 y) {
  return make_double2(fop(sub, c, x.x, y.x), fop(sub, c, x.y, y.y));
}
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ double vadd(double a, double b) { return a + b; }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ double2 vadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float vsub(float a, float b) { return a - b; }
__device__ __forceinline__ double vsub(double a, double b) { return a - b; }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ double2 vsub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ double vmul(double a, double b) { return a * b; }
// Scale multiplies stay two scalar __fmul_rn: the packed multiply may be
// contracted with a following packed add (a unit step right after the scale
// of a reverse-stepping program) into one fused operation, which rounds
// differently from the reference's separate multiply and add.
__device__ __forceinline__ float2 vmul(float2 a, float b) {
  return make_float2(__fmul_rn(a.x, b), __fmul_rn(a.y, b));
}
__device__ __forceinline__ double2 vmul(double2 a, double b) {
  return make_double2(a.x * b, a.y * b);
}
template <typename VT>
__device__ __forceinline__ VT vzero() {
  return VT{};
}
template <typename T>
__device__ __forceinline__ T vlane(const T& v, int) { return v; }
__device__ __forceinline__ float vlane(const float2& v, int k) { return k ? v.y : v.x; }
__device__ __forceinline__ double vlane(const double2& v, int k) { return k ? v.y : v.x; }

}  // namespace lw
