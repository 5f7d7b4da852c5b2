// Overlapped launches (programmatic dependent launch): a kernel launched
// with the programmatic-serialization attribute may be scheduled before the
// kernel ahead of it in the stream has finished, once every CTA of that
// kernel has signalled (griddepcontrol.launch_dependents) or exited.  Each
// kernel launched this way starts with griddepcontrol.wait, which returns
// only when the kernels it depends on have completed and their memory
// operations are visible, and touches no global memory before it; its CTAs
// only get their launch and prologue (shared memory set-up) done early.
// The hardware orders the wait: no flag is polled.
//
// Launches enqueued directly on a stream use it (back-to-back transform
// calls: 4096^2 float32 CDF 9/7 forward + adjoint, four calls, 140 -> 132
// us on a B200); launches recorded into a CUDA graph by stream capture do
// not, since the replayed graph measured slower with it (128 -> 134 us).
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace lw {

// Whether launches use the attribute (the "overlap_launches" option).
bool pdl_enabled();
// Whether launches recorded by stream capture use it too (the
// "overlap_in_graphs" option: 0 none, 1 every launch, 2 the TMA-staged
// strided kernel's launches only); kind 1 marks those launches.
bool pdl_in_graphs(int kind);

template <typename... KArgs, typename... Args>
cudaError_t launch_overlapped_kind(int kind, void (*kern)(KArgs...), int grid, int block,
                                   size_t smem, cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
    cudaGetLastError();  // clear it: the launch below reports its own
    cap = cudaStreamCaptureStatusActive;
  }
  cfg.numAttrs =
      (pdl_enabled() && (cap == cudaStreamCaptureStatusNone || pdl_in_graphs(kind))) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <typename... KArgs, typename... Args>
cudaError_t launch_overlapped(void (*kern)(KArgs...), int grid, int block, size_t smem,
                              cudaStream_t stream, Args&&... args) {
  return launch_overlapped_kind(0, kern, grid, block, smem, stream, std::forward<Args>(args)...);
}

#ifdef __CUDACC__
// Waits for the kernels this one depends on (a no-op without the attribute).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the next kernel in the stream be scheduled once every CTA of this
// one has signalled or exited.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#endif

}  // namespace lw
