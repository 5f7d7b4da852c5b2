// Public vocabulary of the drop-in C++ API: the enums (same names and
// values as the reference's src/lifted-common.hpp:33-125, because callers
// pass them by value and pylifted maps names to them), the shape/stride
// vector types (:105-107) and max_level (:1099-1115).
//
// The X-macro lists keep the reference's names so that code which expands
// them compiles unchanged.  Unlike the header-only reference, the wavelet
// list of this precompiled library is fixed; user-defined step programs go
// through lifted_lwt_sep_program_* in lifted_capi.h instead.
#ifndef LIFTED_COMMON_H_
#define LIFTED_COMMON_H_

#include <cstddef>
#include <cstdint>
#include <vector>

#ifndef LIFTED_WAVELETS
#define LIFTED_WAVELETS \
  X(Lazy, 0)            \
  X(Daubechies1, 1)     \
  X(Daubechies2, 2)     \
  X(Daubechies3, 3)     \
  X(Daubechies4, 4)     \
  X(Daubechies5, 5)     \
  X(Daubechies6, 6)     \
  X(Daubechies7, 7)     \
  X(Daubechies8, 8)     \
  X(Daubechies9, 9)     \
  X(Daubechies10, 10)   \
  X(Symlet4, 104)       \
  X(Symlet5, 105)       \
  X(Symlet6, 106)       \
  X(Coiflet2, 202)      \
  X(Coiflet3, 203)      \
  X(Bior1_3, 10103)     \
  X(Bior1_5, 10105)     \
  X(Bior2_2, 10202)     \
  X(Bior2_4, 10204)     \
  X(Bior2_6, 10206)     \
  X(Bior2_8, 10208)     \
  X(Bior3_1, 10301)     \
  X(Bior3_3, 10303)     \
  X(Bior3_5, 10305)     \
  X(Bior3_7, 10307)     \
  X(Bior3_9, 10309)     \
  X(Bior4_2, 10402)     \
  X(Bior4_4, 10404)     \
  X(Bior4_6, 10406)     \
  X(Bior5_5, 10505)     \
  X(Bior6_8, 10608)     \
  X(CDF5_3, 100503)     \
  X(CDF9_7, 100907)
#endif

#ifndef LIFTED_BOUNDARY_CONDITIONS
#define LIFTED_BOUNDARY_CONDITIONS \
  X(Zero, 0)                       \
  X(Constant, 1)                   \
  X(Periodic, 2)                   \
  X(Symmetric, 3)                  \
  X(Reflect, 4)
#endif
#ifndef LIFTED_N_BC_TYPES
#define LIFTED_N_BC_TYPES 5
#endif

#ifndef LIFTED_TRANSFORM_TYPES
#define LIFTED_TRANSFORM_TYPES \
  X(Forward, 0)                \
  X(Inverse, 1)                \
  X(ForwardAdjoint, 2)         \
  X(InverseAdjoint, 3)
#endif
#ifndef LIFTED_N_TRANSFORM_TYPES
#define LIFTED_N_TRANSFORM_TYPES 4
#endif

namespace lifted {

using std::ptrdiff_t;
using std::size_t;

using size_v = std::vector<size_t>;
using stride_v = std::vector<ptrdiff_t>;
using stride_t = stride_v::value_type;

enum class Wavelet : std::uint32_t {
#define X(name, val) name = val,
  LIFTED_WAVELETS
#undef X
};

enum class BoundaryCondition : std::uint32_t {
#define X(name, val) name = val,
  LIFTED_BOUNDARY_CONDITIONS
#undef X
};

enum class Transform : std::uint32_t {
#define X(name, val) name = val,
  LIFTED_TRANSFORM_TYPES
#undef X
};

// Levels of a width-`width` wavelet on length n: count halvings while
// n >= 2 * (width - 1).  The reference loops forever for width 1; this
// returns (size_t)-1 there.
inline size_t max_level(const size_t width, size_t n) {
  if (width == 0) return 0;
  if (width == 1) return static_cast<size_t>(-1);
  if (n < width - 1) return 0;
  size_t lvl = 0;
  while (n >= 2 * (width - 1)) {
    lvl += 1;
    n = (n + 1) / 2;
  }
  return lvl;
}

// max_level over the transformed axes (the reference reads axes[i] for
// i < shape.size(); this takes the minimum over the axes given).
inline size_t max_level(const size_t width, const size_v& shape,
                        const size_v& axes) {
  if (axes.empty()) return 0;
  size_t min_n = shape[axes[0]];
  for (size_t i = 1; i < axes.size(); ++i)
    if (shape[axes[i]] < min_n) min_n = shape[axes[i]];
  return max_level(width, min_n);
}

}  // namespace lifted

#endif  // LIFTED_COMMON_H_
