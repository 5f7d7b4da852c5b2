// Host-side interfaces of the B200 lifting DWT library.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/lifted_capi.h"
#include "lw_types.hpp"

namespace lw {

// One catalogue or user step with its coefficients as long double, exactly
// as the reference's step factories see them before the cast to T.
struct StepRow {
  int kind, target, offset, ntaps, pm;
  long double c[MAX_TAPS];
};

struct Program {
  std::vector<StepRow> rows;
  size_t width = 0;     // used by max_level (level 0)
  int cat_index = -1;   // catalogue position; -1 for user programs
};

// Per-call knobs of the axis passes.
struct PassOptions {
  bool force_global = false;   // line buffers in global scratch even if the
                               // line fits in shared memory (testing)
  int max_global_ctas = 296;   // CTAs of the global-scratch path
  void* scratch = nullptr;     // caller-provided scratch (else allocated)
  size_t scratch_bytes = 0;
  bool no_alloc = false;       // refuse anything that would allocate
  bool fast_path = true;       // use the register-blocked kernels when they apply
};

int set_error(int status, const char* fmt, ...);
void clear_error();
void count_launches(uint64_t n);
// Launches per kernel family, for tests that check which kernel a pass ran
// on (lifted_kernel_launch_count).
enum KernelFamily {
  KF_LINE, KF_REG, KF_WROW, KF_WROW2, KF_WTILE, KF_COL, KF_BATCH, KF_COPY, KF_BLUR,
  KF_COUNT
};
void count_family(int fam, uint64_t n);
uint64_t family_count(int fam);
int family_index(const char* name);
// L2 priority code (lw_cache.cuh) of the fast kernels' loads and stores:
// evict_first loads and evict_last stores when the "l2_hints" option is on.
int l2_hint_code();
// The reference's boundary index maps (src/lifted-common.hpp:719-779) on the
// host, for inputs on which its loops terminate; n means "skip the tap".
int64_t host_bc_index(int bc, int64_t i, int64_t n);
const char* last_error();
uint64_t launch_count();

PassOptions default_options();
int set_option(const char* name, int64_t value);

int catalogue_program(uint32_t wavelet, Program* prog);
int user_program(const lifted_step_t* steps, size_t nsteps, size_t width,
                 Program* prog);
template <typename T>
void resolve_program(const Program& prog, int op, int across,
                     DevProgram<T>* out);

size_t max_level(size_t width, size_t n);
// Device or managed memory (cudaPointerGetAttributes).
bool device_pointer(const void* p);
bool line_degenerate(const Program& prog, int op, int bc, int64_t n,
                     size_t levels);
size_t wavelet_count();
uint32_t wavelet_value(size_t i);
size_t wavelet_width(uint32_t w);

// Runs the lines of an axis pass (contiguous, non-negative offsets) as a
// cached batch plan of the batch engine, one signal per line: 1 done, 0 not
// eligible, -1 failed (the error is set).
// Runs a batch of nD images (dense C-order, each transformed separably over
// all of its axes) as one persistent launch of line items, from a cached
// plan.  Returns a status; *ran is false (and the status LIFTED_OK) when it
// did not run because a new plan would have to be built inside a stream
// capture.
template <typename T>
int run_batch_nd(uint32_t op, uint32_t bc, size_t nimg, const lifted_image_t* ims, const T* in,
                 T* out, cudaStream_t stream, bool* ran);
// The "batch_nd_mode" option: 0 automatic, 1 persistent, 2 grouped.
int batch_nd_mode();
// The "edge_kernels_always" option: Zero passes run the exact-edge kernel
// instantiations too (their edge work then never runs; for comparing the
// two instantiations).
bool edge_kernels_always();
// Whether zero_step (lw_line_kernel.cuh) reproduces the exact step code on
// `levels` levels of a line of length n under boundary bc: the Zero boundary
// and, at every level (bands of ceil(m / 2) and floor(m / 2)), no step whose
// front edge range [0, n1) reaches past the start n2 of its back edge range
// (src/lifted-steps-inl.hpp:409-410; such indices take both updates).
// False as well when the "zero_step_code" option is off.
template <typename T>
bool zero_fast_ok(const DevProgram<T>& prog, int bc, int64_t n, int levels);
// Per-axis levels of the separable driver, resolved and checked (level 0 =
// max_level; degenerate bands refused), as lifted_lwt_sep_* does.
int resolve_sep_levels(const Program& prog, uint32_t op, uint32_t bc,
                       const size_t* shape, size_t naxes, const size_t* axes,
                       const size_t* levels, std::vector<size_t>* lv);

template <typename T>
int run_lines_batched(uint32_t wavelet, int op, int bc, const LineGeom& g, int levels,
                      const T* in, T* out, cudaStream_t stream);

template <typename T>
int lwt_entry(const Program& prog, bool separable, uint32_t op, uint32_t bc,
              size_t ndim, const size_t* shape, const ptrdiff_t* sin,
              const ptrdiff_t* sout, size_t naxes, const size_t* axes,
              const size_t* levels, size_t level, const T* in, T* out,
              void* stream, const PassOptions& opt);

}  // namespace lw
