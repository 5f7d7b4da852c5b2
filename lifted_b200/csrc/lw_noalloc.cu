// The separable transform entry point that allocates nothing.
//
// Some callers must not allocate device memory: for example a host
// application that reserves the GPU's memory for its own allocator and
// forbids its plugins from calling cudaMalloc, or a latency-critical
// processing loop where an allocation's possible implicit synchronisation or
// out-of-memory failure is not acceptable.  lifted_lwt_sep_noalloc_f32 serves
// them: it runs the general line kernel, and when a line is too long for
// shared memory, that kernel's per-CTA line buffers come from one fixed
// array of LIFTED_NOALLOC_SCRATCH_BYTES bytes of static device memory
// defined below (every GPU that loads this library holds it until the
// process exits) instead of from a stream-ordered allocation.
//
// The array's host-side name is only a stand-in for the device address: the
// kernel gets the address from cudaGetSymbolAddress, taken once per device
// with that device current, on the first call on the device.  With lazy
// module loading (the CUDA default since 12.2) that first call is also when
// the module loads and the array's memory is reserved on the device, so make
// the first call on each device early: before the host application claims
// the GPU's memory for its own allocator, and before any stream capture (or
// set CUDA_MODULE_LOADING=EAGER, which reserves it when the library's
// kernels load).
//
// The options of lifted_set_option apply (the general kernel's CTA count
// among them), except that the fast kernels are never used: they take their
// scratch from stream-ordered allocations.
//
// Every call shares the array and it keeps the last call's contents.  The
// kernel writes every scratch element before reading it, so nothing needs
// clearing between calls; but calls whose kernels overlap on the GPU (two
// streams, or two host threads) race on the array and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/lifted_capi.h"
#include "lw_host.hpp"
#include "lw_launch.hpp"

namespace lw {
namespace {

static __device__ __align__(256) unsigned char
    g_noalloc_scratch[LIFTED_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the static scratch on the current device (set-up on the
// first call per device).
int noalloc_scratch(void** ptr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return set_error(LIFTED_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(LIFTED_EINVAL, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(LIFTED_ECUDA, "cudaGetSymbolAddress(scratch): %s",
                       cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *ptr = g_noalloc_ptr[dev];
  return LIFTED_OK;
}

}  // namespace
}  // namespace lw

extern "C" LIFTED_CAPI int lifted_lwt_sep_noalloc_f32(
    uint32_t wavelet, uint32_t op, uint32_t bc, size_t ndim,
    const size_t* shape, const ptrdiff_t* stride_in,
    const ptrdiff_t* stride_out, size_t naxes, const size_t* axes,
    const size_t* levels, const float* in, float* out, void* stream) {
  lw::clear_error();
  lw::Program prog;
  int rc = lw::catalogue_program(wavelet, &prog);
  if (rc) return rc;
  void* scratch = nullptr;
  rc = lw::noalloc_scratch(&scratch);
  if (rc) return rc;
  // in and out must live on the current device: the scratch array used is
  // this device's copy.
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess)
    return lw::set_error(LIFTED_ECUDA, "cudaGetDevice failed");
  for (const void* ptr : {(const void*)in, (const void*)out}) {
    if (!ptr) continue;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
      cudaGetLastError();
      continue;  // host memory: refused below with LIFTED_EINVAL
    }
    if ((at.type == cudaMemoryTypeDevice) && at.device != dev)
      return lw::set_error(LIFTED_EINVAL,
                           "pointer %p is on device %d, the current device is %d", ptr,
                           at.device, dev);
  }
  lw::PassOptions opt = lw::default_options();
  opt.no_alloc = true;
  opt.fast_path = false;
  opt.scratch = scratch;
  opt.scratch_bytes = LIFTED_NOALLOC_SCRATCH_BYTES;
  return lw::lwt_entry<float>(prog, true, op, bc, ndim, shape, stride_in,
                              stride_out, naxes, axes, levels, 0, in, out,
                              stream, opt);
}
