// L2 eviction priorities of the fast kernels' global loads and stores.
//
// A separable transform runs one full pass per axis (the reference's
// general_nd, src/lifted-drivers-inl.hpp:459-485), and each later pass
// reads what the previous one wrote.  An image of up to a few tens of MiB
// fits in the B200's L2 (126 MB), so the passes can hand their result to the
// next through L2 instead of DRAM if what was just written outlives what was
// just read: a pass reads its input with evict_first (it is consumed) and
// writes its output with evict_last (the next pass, or the caller, reads it
// next).  Per-instruction policies (createpolicy + .L2::cache_hint) only;
// nothing is set aside or changed device-wide.
//
// A priority code packs both: bits 0-1 the loads', bits 2-3 the stores'
// (L2_NORMAL, L2_FIRST, L2_LAST).
#pragma once

#include <cstdint>

namespace lw {

enum L2Prio { L2_NORMAL = 0, L2_FIRST = 1, L2_LAST = 2 };

constexpr int l2_code(int load, int store) { return (load & 3) | ((store & 3) << 2); }

#ifdef __CUDACC__

__device__ __forceinline__ uint64_t l2_policy(int prio) {
  uint64_t pol;
  if (prio == L2_FIRST)
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  else if (prio == L2_LAST)
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  else
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint64_t l2_load_policy(int code) { return l2_policy(code & 3); }
__device__ __forceinline__ uint64_t l2_store_policy(int code) {
  return l2_policy((code >> 2) & 3);
}

// Stores with an L2 cache policy.
__device__ __forceinline__ void st_hint(float* p, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_hint(double* p, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_hint(float* p, float2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x),
               "f"(v.y), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_hint(double* p, double2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v.x),
               "d"(v.y), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_hint(float* p, float4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p),
               "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol)
               : "memory");
}

// 16-byte asynchronous copy global -> shared with an L2 cache policy.
__device__ __forceinline__ void cp_async16_hint(unsigned saddr, const void* src, uint64_t pol) {
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(saddr),
               "l"(src), "l"(pol)
               : "memory");
}

#endif  // __CUDACC__

}  // namespace lw
