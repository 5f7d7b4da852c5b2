/* C ABI of the B200 lifting-scheme DWT library (liblifted_b200.so).
 *
 * This is the device boundary of the drop-in: the C++ overloads of
 * lifted::lwt in lifted.hpp and the Python package lifted_b200 (pylifted
 * API) both call these functions.  Plain pointers and sizes only; no
 * exceptions cross this boundary and nothing here aborts.
 *
 * Enum values are the reference's (src/lifted-common.hpp:33-98):
 *   wavelet   lifted::Wavelet            (0 Lazy ... 100907 CDF9_7)
 *   op        lifted::Transform          0 Forward, 1 Inverse,
 *                                        2 ForwardAdjoint, 3 InverseAdjoint
 *   bc        lifted::BoundaryCondition  0 Zero, 1 Constant, 2 Periodic,
 *                                        3 Symmetric, 4 Reflect
 * Shapes are in elements; strides are in elements and may be negative.
 *
 * Pointers: device (or managed) pointers run asynchronously on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) with no hidden
 * synchronisation.  Host pointers are staged: the call copies the spanned
 * input to the GPU, runs, copies the result back and returns after the copy
 * has finished.  `in == out` with identical strides is allowed (in place).
 *
 * Every function returns one of the LIFTED_* status codes below.
 */
#ifndef LIFTED_CAPI_H_
#define LIFTED_CAPI_H_

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define LIFTED_CAPI __declspec(dllexport)
#else
#define LIFTED_CAPI __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define LIFTED_OK 0
/* Invalid argument: unknown wavelet/transform/boundary value, axis >= ndim,
 * unsupported rank, bad step program. */
#define LIFTED_EINVAL 1
/* An input on which the reference hangs, divides by zero or indexes out of
 * bounds: level 0 with the Lazy wavelet (max_level never returns), a
 * Periodic/Symmetric/Reflect boundary evaluated on an empty band, Reflect on
 * a one-element band, the non-separable driver resolving to zero levels.
 * Nothing is written. */
#define LIFTED_EDEGENERATE 2
#define LIFTED_ENOTIMPL 3
/* A CUDA runtime call failed (the message names it). */
#define LIFTED_ECUDA 4
#define LIFTED_ENOMEM 5
/* A bounded device-side wait gave up. */
#define LIFTED_ETIMEOUT 6
/* Request exceeds a stated limit (e.g. the fixed scratch of an entry point
 * that allocates nothing). */
#define LIFTED_ETOOLARGE 7

/* A user-defined lifting step (the runtime counterpart of the reference's
 * compile-time step descriptors, src/lifted-common.hpp:798-1032).
 *   kind     0 generic update (ntaps coefficients in coef[0..ntaps)),
 *            1 unit update (y += x[i+offset] or -=, per unit_sub),
 *            2 repeat update (coef[0] * sum of ntaps neighbours),
 *            3 scale (ntaps 1: coef[0] = s_mul = d_div; ntaps 2: coef[0] =
 *              s_mul, coef[1] = d_div)
 *   target   0 updates the even samples (s), 1 the odd samples (d)
 *   offset   offset of the first tap relative to the updated index
 * Coefficients are given as double; casts to float and the 1/c of scale
 * steps follow the reference (1.0L / c rounded to the element type). */
typedef struct lifted_step {
  uint32_t kind;
  uint32_t target;
  int32_t offset;
  uint32_t ntaps;
  uint32_t unit_sub;
  uint32_t reserved;
  double coef[9];
} lifted_step_t;

#define LIFTED_MAX_TAPS 9
#define LIFTED_MAX_STEPS 32
#define LIFTED_MAX_NDIM 16

/* Separable nD transform: every axis in `axes` (in that order) gets the full
 * levels[i]-level 1D transform; level 0 means max_level(width, length).
 * Replaces lifted::lwt(..., const size_v& levels, const T* ...) for T = float, double
 * (src/lifted.hpp:27-39, src/lifted-sep-float.cpp:20-30,
 * src/lifted-sep-double.cpp:20-30). */
LIFTED_CAPI int lifted_lwt_sep_f32(uint32_t wavelet, uint32_t op, uint32_t bc,
                                   size_t ndim, const size_t* shape,
                                   const ptrdiff_t* stride_in,
                                   const ptrdiff_t* stride_out, size_t naxes,
                                   const size_t* axes, const size_t* levels,
                                   const float* in, float* out, void* stream);
LIFTED_CAPI int lifted_lwt_sep_f64(uint32_t wavelet, uint32_t op, uint32_t bc,
                                   size_t ndim, const size_t* shape,
                                   const ptrdiff_t* stride_in,
                                   const ptrdiff_t* stride_out, size_t naxes,
                                   const size_t* axes, const size_t* levels,
                                   const double* in, double* out,
                                   void* stream);

/* Non-separable (Mallat) nD transform: `level` levels, each a single-level
 * transform of every axis over the shrinking approximation corner; level 0
 * means max_level over the transformed axes.
 * Replaces lifted::lwt(..., const size_t level, const T* ...) for T = float, double
 * (src/lifted.hpp:13-25, src/lifted-float.cpp:20-30,
 * src/lifted-double.cpp:20-30). */
LIFTED_CAPI int lifted_lwt_f32(uint32_t wavelet, uint32_t op, uint32_t bc,
                               size_t ndim, const size_t* shape,
                               const ptrdiff_t* stride_in,
                               const ptrdiff_t* stride_out, size_t naxes,
                               const size_t* axes, size_t level,
                               const float* in, float* out, void* stream);
LIFTED_CAPI int lifted_lwt_f64(uint32_t wavelet, uint32_t op, uint32_t bc,
                               size_t ndim, const size_t* shape,
                               const ptrdiff_t* stride_in,
                               const ptrdiff_t* stride_out, size_t naxes,
                               const size_t* axes, size_t level,
                               const double* in, double* out, void* stream);

/* Separable transform with a caller-supplied step program in place of a
 * catalogue wavelet (the reference selects its wavelet list at compile time
 * through the overridable LIFTED_WAVELETS X-macro, src/lifted-common.hpp:33;
 * a precompiled GPU library takes the program at run time instead).  `width`
 * is only used when a level is 0.  Steps run in the given order for Forward
 * and InverseAdjoint and reversed for Inverse and ForwardAdjoint. */
LIFTED_CAPI int lifted_lwt_sep_program_f32(
    const lifted_step_t* steps, size_t nsteps, size_t width, uint32_t op,
    uint32_t bc, size_t ndim, const size_t* shape, const ptrdiff_t* stride_in,
    const ptrdiff_t* stride_out, size_t naxes, const size_t* axes,
    const size_t* levels, const float* in, float* out, void* stream);
LIFTED_CAPI int lifted_lwt_sep_program_f64(
    const lifted_step_t* steps, size_t nsteps, size_t width, uint32_t op,
    uint32_t bc, size_t ndim, const size_t* shape, const ptrdiff_t* stride_in,
    const ptrdiff_t* stride_out, size_t naxes, const size_t* axes,
    const size_t* levels, const double* in, double* out, void* stream);

/* Separable float32 transform that allocates nothing (no counterpart in the
 * reference, whose CPU transform allocates per-thread line buffers).  For
 * callers that must not allocate device memory -- a host application that
 * reserves the GPU's memory for its own allocator and forbids its plugins
 * from calling cudaMalloc, or a latency-critical loop where an allocation's
 * implicit synchronisation or failure is unacceptable.  Arguments and
 * results as lifted_lwt_sep_f32, with these differences:
 *   - in and out must be device (or managed) pointers; host pointers would
 *     need staging buffers and are rejected with LIFTED_EINVAL;
 *   - lines too long for shared memory are buffered in one static device
 *     array of LIFTED_NOALLOC_SCRATCH_BYTES bytes (held by every GPU that
 *     loads the library until exit); a line longer than that array can hold
 *     (LIFTED_NOALLOC_SCRATCH_BYTES / 6 float32 elements, about 5.6 million)
 *     is rejected with LIFTED_ETOOLARGE;
 *   - the first call on a device looks up the array's device address; with
 *     lazy module loading (the CUDA default) that is also when the module
 *     loads and the array's memory is reserved on the device, so make the
 *     first call before the application takes the GPU's memory and before
 *     any stream capture (or run with CUDA_MODULE_LOADING=EAGER);
 *   - in and out must be on the current device (else LIFTED_EINVAL);
 *   - lifted_set_option settings apply, but the fast kernels are never used
 *     (they allocate scratch), so this entry point serves the general kernel;
 *   - every call shares the array: calls whose kernels overlap on the GPU
 *     (two streams, two host threads) race and must be serialised. */
#define LIFTED_NOALLOC_SCRATCH_BYTES (32u << 20)
LIFTED_CAPI int lifted_lwt_sep_noalloc_f32(
    uint32_t wavelet, uint32_t op, uint32_t bc, size_t ndim,
    const size_t* shape, const ptrdiff_t* stride_in,
    const ptrdiff_t* stride_out, size_t naxes, const size_t* axes,
    const size_t* levels, const float* in, float* out, void* stream);

/* ------------------------------------------------------------------------
 * Batched uneven-length 1D transforms.
 *
 * The reference transforms one array per call (lifted::lwt,
 * src/lifted.hpp:13-39); a batch of signals of different lengths, wavelets
 * and level counts is a loop of such calls (src/pylifted/_wavelets.pyx:
 * 185-276 per call).  Here a batch is one persistent kernel launch that pulls
 * work items (a whole signal, or a tile of a long signal's band over a group
 * of levels) from a device queue.  Each signal's result is that of the
 * separable transform of the 1D array alone:
 *     lifted_lwt_sep_xxx(wavelet, op, bc, 1, {length}, {1}, {1}, 1, {0},
 *                        {levels}, in + in_offset, out + out_offset, stream)
 * Signals are contiguous (unit stride) in `in` and `out`, which must be
 * device (or managed) memory and must not overlap each other.  Signals may
 * share input but their output ranges must be disjoint. */
typedef struct lifted_signal {
  uint32_t wavelet;     /* lifted::Wavelet value */
  uint32_t levels;      /* levels; 0 = max_level(width, length) */
  uint64_t length;      /* samples (0: the signal is skipped) */
  uint64_t in_offset;   /* element offset of the signal in `in` */
  uint64_t out_offset;  /* element offset of its result in `out` */
} lifted_signal_t;

/* Batched nD images (no single counterpart in the reference: a loop of
 * lifted::lwt calls, src/lifted.hpp:13-39, one per image).  Each image is a
 * dense C-order array of ndim (1..4) axes, transformed separably over all of
 * them, in order, exactly as
 *     lifted_lwt_sep_xxx(wavelet, op, bc, ndim, shape, dense strides, ndim,
 *                        {0, .., ndim-1}, levels, in + in_offset,
 *                        out + out_offset, stream)
 * would.  Consecutive entries with the same wavelet, shape and levels whose
 * data lie back to back in both buffers run as one call over a (group,
 * shape...) view.  Device pointers; outputs must be disjoint and no image's
 * output may overlap another image's input (an image may be in place).
 * Stream-ordered, no synchronisation; on an error, the groups before the
 * failing one have been enqueued. */
typedef struct lifted_image {
  uint32_t wavelet;     /* lifted::Wavelet value */
  uint32_t ndim;        /* 1..4 */
  uint64_t shape[4];    /* C order, slowest axis first; entries >= ndim unused */
  uint32_t levels[4];   /* levels per axis; 0 = max_level(width, length) */
  uint64_t in_offset;   /* element offset of the image in `in` */
  uint64_t out_offset;  /* element offset of its result in `out` */
} lifted_image_t;
LIFTED_CAPI int lifted_lwt_batch_nd_f32(uint32_t op, uint32_t bc, size_t nimages,
                                        const lifted_image_t* images, const float* in,
                                        float* out, void* stream);
LIFTED_CAPI int lifted_lwt_batch_nd_f64(uint32_t op, uint32_t bc, size_t nimages,
                                        const lifted_image_t* images, const double* in,
                                        double* out, void* stream);

/* Optional planner settings (0 = default or autotuned):
 *   block        threads per CTA of the persistent kernel (64..512)
 *   whole_max    longest band transformed as one whole item in shared
 *                memory (default 4096 float32, 2048 float64)
 *   tile         interior width of a tile item, samples of its band
 *   tile_levels  levels per tile group (Zero boundary only)
 *   spin_limit   polls of a completion counter before an item that waits
 *                for another item's band gives up (records LIFTED_ETIMEOUT
 *                for lifted_batch_check, skips its work and lets its own
 *                dependents proceed): 0 = default (4 M polls, about a
 *                second), > 0 = that many, < 0 = none, so every waiting
 *                item gives up at once (failure-detection tests) */
typedef struct lifted_batch_tuning {
  uint32_t block;
  uint32_t whole_max;
  uint32_t tile;
  uint32_t tile_levels;
  int32_t spin_limit;
} lifted_batch_tuning_t;

typedef struct lifted_batch_info {
  uint64_t nsignals, nitems, ntiles, nwhole, nwhole_global, ncounters;
  uint64_t scratch_bytes, shared_bytes;
  uint32_t grid, block;
} lifted_batch_info_t;

typedef struct lifted_batch_plan lifted_batch_plan_t;

/* Plans a batch: validates every signal (as the separable entry would),
 * resolves its levels, cuts it into work items, allocates the plan's device
 * buffers (work queue, programs, completion counters, scratch bands).  Tile
 * width and levels per tile group come from `tuning`, else from the
 * autotuner's table for (wavelet, dtype, transform, length), else from a
 * halo-based default. */
LIFTED_CAPI int lifted_batch_plan_create_f32(uint32_t op, uint32_t bc, size_t nsignals,
                                             const lifted_signal_t* signals,
                                             const lifted_batch_tuning_t* tuning,
                                             lifted_batch_plan_t** plan);
LIFTED_CAPI int lifted_batch_plan_create_f64(uint32_t op, uint32_t bc, size_t nsignals,
                                             const lifted_signal_t* signals,
                                             const lifted_batch_tuning_t* tuning,
                                             lifted_batch_plan_t** plan);
/* A reusable plan of a batch of nD images (the lifted_image_t table that
 * lifted_lwt_batch_nd_* takes; no counterpart in the reference, whose batch
 * is a loop of lwt calls, src/pylifted/_wavelets.pyx:185-264): one
 * persistent launch per run; every (image, axis) pass is cut into line
 * items of whole lines on the device queue, and the items of an image's
 * later axes wait (bounded) on a completion counter of its earlier axes.
 * Run, replay, check, inspect and destroy it with the lifted_batch_* calls.
 * in == out is allowed when every image's input offset equals its output
 * offset or its input meets no output.  Tuning: whole_max sets the shared
 * memory per CTA (1.5 * whole_max elements; longer lines work in a global
 * slot per CTA), block the CTA size, spin_limit as below; tile and
 * tile_levels are unused. */
LIFTED_CAPI int lifted_batch_plan_create_nd_f32(uint32_t op, uint32_t bc, size_t nimages,
                                                const lifted_image_t* images,
                                                const lifted_batch_tuning_t* tuning,
                                                lifted_batch_plan_t** plan);
LIFTED_CAPI int lifted_batch_plan_create_nd_f64(uint32_t op, uint32_t bc, size_t nimages,
                                                const lifted_image_t* images,
                                                const lifted_batch_tuning_t* tuning,
                                                lifted_batch_plan_t** plan);
/* Enqueues one run on `stream` (a memset of the queue counters and one
 * kernel launch; stream-ordered, no synchronisation, may be captured into a
 * CUDA graph).  Runs of one plan must not overlap on the GPU. */
LIFTED_CAPI int lifted_batch_run(lifted_batch_plan_t* plan, const void* in, void* out,
                                 void* stream);
/* As lifted_batch_run, replayed from a CUDA graph the plan captures on first
 * use (and again whenever `in` or `out` change). */
LIFTED_CAPI int lifted_batch_run_graph(lifted_batch_plan_t* plan, const void* in, void* out,
                                       void* stream);
/* Synchronises `stream` and reports LIFTED_ETIMEOUT if an item of the last
 * run gave up waiting (bounded) for the band another item produces. */
LIFTED_CAPI int lifted_batch_check(lifted_batch_plan_t* plan, void* stream);
LIFTED_CAPI int lifted_batch_plan_info(const lifted_batch_plan_t* plan,
                                       lifted_batch_info_t* info);
/* Fields of work item `index` in queue order: kind, program, signal, lev0,
 * nlev, src_sel, dst_sel, wait_ctr, wait_target, done_ctr, n0, in_off,
 * out_off, src_off, dst_off, t0, t1, halo, gbuf, phase, geo (for tests and
 * diagnostics). */
LIFTED_CAPI int lifted_batch_plan_item(const lifted_batch_plan_t* plan, size_t index,
                                       int64_t* fields, size_t nfields);
/* Axis-pass geometry `index` of a plan of nD images (the `geo` field of its
 * line items): line length, element stride along the axis, the other three
 * dims fastest first (1 where absent) and their element strides. */
LIFTED_CAPI int lifted_batch_plan_geo(const lifted_batch_plan_t* plan, size_t index,
                                      int64_t* fields, size_t nfields);
LIFTED_CAPI void lifted_batch_plan_destroy(lifted_batch_plan_t* plan);
/* One-shot: plan, run, check, destroy (synchronous). */
LIFTED_CAPI int lifted_lwt_batch_f32(uint32_t op, uint32_t bc, size_t nsignals,
                                     const lifted_signal_t* signals, const float* in,
                                     float* out, void* stream);
LIFTED_CAPI int lifted_lwt_batch_f64(uint32_t op, uint32_t bc, size_t nsignals,
                                     const lifted_signal_t* signals, const double* in,
                                     double* out, void* stream);
/* Autotuner: for each wavelet, times every (tile width, levels per tile
 * group) candidate on a synthetic batch of `total` samples cut into signals
 * of `length`, and records the fastest in the process-wide table keyed by
 * (wavelet, dtype, transform, log2 length, stride 1) that later plans
 * consult.  Allocates its own device buffers. */
LIFTED_CAPI int lifted_batch_autotune(uint32_t dtype_bytes, uint32_t op, uint32_t bc,
                                      size_t nwavelets, const uint32_t* wavelets,
                                      size_t length, size_t total, void* stream);
/* The tuning table as JSON (one entry per line), and back. */
LIFTED_CAPI int lifted_batch_tune_save(const char* path);
LIFTED_CAPI int lifted_batch_tune_load(const char* path, size_t* loaded);
LIFTED_CAPI void lifted_batch_tune_clear(void);

/* max_level(width, n) of the reference (src/lifted-common.hpp:1099-1108);
 * returns (size_t)-1 for width 1, where the reference never returns. */
LIFTED_CAPI size_t lifted_max_level(size_t width, size_t n);
/* `width` of a catalogue wavelet (src/lifted-wavelets.hpp), 0 if unknown. */
LIFTED_CAPI size_t lifted_wavelet_width(uint32_t wavelet);
/* Number of catalogue wavelets and the enum value of the i-th. */
LIFTED_CAPI size_t lifted_wavelet_count(void);
LIFTED_CAPI uint32_t lifted_wavelet_value(size_t index);
/* Static description of a status code. */
LIFTED_CAPI const char* lifted_status_string(int status);
/* Detail of the last failure on the calling thread ("" if none). */
LIFTED_CAPI const char* lifted_last_error(void);
/* Number of kernel launches this library has issued from the calling
 * process (for instrumentation). */
LIFTED_CAPI uint64_t lifted_launch_count(void);
/* Launches of one kernel family since the process started (for tests that
 * check which kernel served a pass; no counterpart in the reference):
 * "line" (the exact general kernel), "reg", "wrow", "wrow2", "wtile",
 * "col" (the TMA-staged strided kernel), "batch", "copy", "blur".  0 for an
 * unknown name. */
LIFTED_CAPI uint64_t lifted_kernel_launch_count(const char* family);
/* Process-wide tuning/testing knobs:
 *   "force_global_scratch" 0/1  keep line buffers in global scratch even
 *                               when a line fits in shared memory
 *   "max_global_ctas"      n    CTAs of the global-scratch line path
 *   "fast_path"            0/1  register-blocked kernels where they apply
 *   "tma_strided"          0/1  TMA-staged kernel for strided float32 passes
 *   "tma_packed"           0/1  two adjacent lines per lane in that kernel
 *   "tma_stacked"          0/1  strided lines of 32..256 samples in a 3D
 *                               view: one staging window holds 512/n
 *                               consecutive outer slices
 *   "long_lines_batched"   0/1  contiguous lines too long for one CTA run
 *                               on the batch engine (many CTAs per line)
 *   "wrow_split"           0/1  float32 rows of 2048/4096 split over two
 *                               warps (else one warp per row)
 *   "generic_kernels"      0/1  catalogue wavelets without compiled kernels
 *                               run on the generic register kernels (each
 *                               step dispatched on its shape) where they
 *                               apply (else the general line kernel)
 *   "row_windows"          0/1  contiguous rows longer than one warp holds
 *                               run every level on windows with halos,
 *                               one warp each (else the batch engine)
 *   "overlap_launches"     0/1  programmatic dependent launch: the next
 *                               transform kernel in a stream is scheduled
 *                               while the one before it drains, and waits
 *                               in hardware for its results (launches
 *                               recorded by stream capture never use it)
 *   "l2_hints"             0/1  fast kernels read with L2 evict_first and
 *                               write with evict_last (per-instruction
 *                               cache policies; off: measured no gain)
 *   "col_row_order"        0/1  the TMA-staged strided kernel takes its
 *                               tiles row tile by row tile (neighbouring
 *                               CTAs read neighbouring strips of the same
 *                               rows; else strip by strip)
 *   "batch_nd_mode"        0..2 batches of nD images: 0 automatic, 1 one
 *                               persistent launch of line items, 2 one
 *                               separable call per group of identically
 *                               shaped, packed images
 *   "zero_step_code"       0/1  Zero-boundary passes on the general line
 *                               kernel and the batch engine's whole and
 *                               line items sum each update's in-band taps
 *                               directly (same results; else the exact
 *                               step code with its boundary map)
 *   "edge_kernels_always"  0/1  Zero passes run the exact-edge kernel
 *                               instantiations too (for comparing them)
 *   "overlap_in_graphs"    0..2 programmatic dependent launch inside
 *                               stream captures: 0 never, 1 always, 2 the
 *                               TMA-staged strided kernel only */
LIFTED_CAPI int lifted_set_option(const char* name, int64_t value);
/* Synchronises `stream` and reports LIFTED_ETIMEOUT if a kernel of this
 * library gave up a bounded device-side wait since the last check (the
 * affected output is not valid).  Clears the condition. */
LIFTED_CAPI int lifted_device_check(void* stream);

/* Blur operator of the wavelet-regularised least-squares form (no
 * counterpart in the reference, which has no solver): 2D correlation of each
 * of `nimg` contiguous h x w float32 images with a k x k kernel (odd k <= 7,
 * row-major host array), zero padding, same size; adjoint != 0 correlates
 * with the flipped kernel (the transpose).  Device pointers, no overlap,
 * stream-ordered. */
LIFTED_CAPI int lifted_blur2d_f32(const float* in, float* out, size_t nimg, size_t h, size_t w,
                                  const float* kernel, size_t k, int adjoint, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LIFTED_CAPI_H_ */
