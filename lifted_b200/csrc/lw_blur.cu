// 2D correlation with a small odd kernel (zero padding, "same" size) over a
// batch of float32 images: the blur operator A of the wavelet-regularised
// least-squares loop (lifted_b200/lsq.py) and its adjoint A^T (correlation
// with the flipped kernel).  Not part of the reference; it replaces a
// library convolution whose backward pass ran a TF32 implicit GEMM (a
// precision loss in the gradient and 17 ms per call on 16 x 2048^2).
//
// One CTA (256 threads: 64 columns x 4 row groups) computes a 32 x 64
// output tile of one image: the tile plus its (K-1)/2 margin is staged in
// shared memory (zero outside the image), then each thread runs 8 output
// rows of one column, summing the
// K x K products in a fixed order (kernel rows outer, columns inner, one
// fused multiply-add each).  HBM-bound: one read and one write of the batch.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>

#include "lifted_capi.h"
#include "lw_host.hpp"
#include "lw_pdl.hpp"

namespace lw {
namespace {

constexpr int BLUR_MAXK = 7;
constexpr int BLUR_TW = 64;   // tile columns (one thread each)
constexpr int BLUR_TH = 32;   // tile rows
constexpr int BLUR_TY = 4;    // row groups per column
constexpr int BLUR_RPT = BLUR_TH / BLUR_TY;  // rows per thread

struct BlurParams {
  const float* in;
  float* out;
  int64_t h, w;        // image size
  int64_t tiles_x, tiles_y;
  int32_t k;           // kernel size (odd, <= BLUR_MAXK)
  int32_t pad_;
  float wts[BLUR_MAXK * BLUR_MAXK];  // row-major, already flipped for A^T
};

template <int K>
__global__ void __launch_bounds__(BLUR_TW * BLUR_TY)
    blur_kernel(const __grid_constant__ BlurParams p) {
  constexpr int R = K / 2;
  constexpr int SW = BLUR_TW + K - 1, SH = BLUR_TH + K - 1;
  __shared__ float tile[SH][SW + 1];
  pdl_wait();
  pdl_trigger();
  const int64_t per_img = p.tiles_x * p.tiles_y;
  const int64_t img = blockIdx.x / per_img;
  const int64_t t = blockIdx.x - img * per_img;
  const int64_t ty0 = (t / p.tiles_x) * BLUR_TH;
  const int64_t tx0 = (t % p.tiles_x) * BLUR_TW;
  const float* src = p.in + img * p.h * p.w;
  const int tid = threadIdx.x;
  const int tcol = tid % BLUR_TW, trow = tid / BLUR_TW;  // column, row group
  for (int e = tid; e < SH * SW; e += BLUR_TW * BLUR_TY) {
    const int r = e / SW, c = e - r * SW;
    const int64_t y = ty0 + r - R, x = tx0 + c - R;
    tile[r][c] = (y >= 0 && y < p.h && x >= 0 && x < p.w) ? src[y * p.w + x] : 0.0f;
  }
  __syncthreads();
  float wk[K * K];
#pragma unroll
  for (int i = 0; i < K * K; ++i) wk[i] = p.wts[i];
  const int c = tcol;
  const int64_t x = tx0 + c;
  float* dst = p.out + img * p.h * p.w;
#pragma unroll
  for (int rr = 0; rr < BLUR_RPT; ++rr) {
    const int r = trow * BLUR_RPT + rr;
    float acc = 0.0f;
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
      for (int j = 0; j < K; ++j) acc = __fmaf_rn(wk[i * K + j], tile[r + i][c + j], acc);
    const int64_t y = ty0 + r;
    if (y < p.h && x < p.w) dst[y * p.w + x] = acc;
  }
}

template <int K>
cudaError_t launch_blur(const BlurParams& p, int64_t grid, cudaStream_t stream) {
  return launch_overlapped(blur_kernel<K>, (int)grid, BLUR_TW * BLUR_TY, 0, stream, p);
}

}  // namespace
}  // namespace lw

extern "C" {

LIFTED_CAPI int lifted_blur2d_f32(const float* in, float* out, size_t nimg, size_t h, size_t w,
                                  const float* kernel, size_t k, int adjoint, void* stream) {
  using namespace lw;
  clear_error();
  if (!in || !out || !kernel) return set_error(LIFTED_EINVAL, "null pointer");
  if (k < 1 || k > (size_t)BLUR_MAXK || (k % 2) == 0)
    return set_error(LIFTED_EINVAL, "kernel size %zu: odd and at most %d", k, BLUR_MAXK);
  if (nimg == 0 || h == 0 || w == 0) return LIFTED_OK;
  if (!device_pointer(in) || !device_pointer(out))
    return set_error(LIFTED_EINVAL, "in and out must be device pointers");
  const size_t total = nimg * h * w;
  if (total / nimg / h != w) return set_error(LIFTED_EINVAL, "size overflow");
  const char* ib = (const char*)in;
  const char* ob = (const char*)out;
  if (ib < ob + total * sizeof(float) && ob < ib + total * sizeof(float))
    return set_error(LIFTED_EINVAL, "in and out overlap");
  BlurParams p;
  std::memset(&p, 0, sizeof(p));
  p.in = in;
  p.out = out;
  p.h = (int64_t)h;
  p.w = (int64_t)w;
  p.tiles_x = ((int64_t)w + BLUR_TW - 1) / BLUR_TW;
  p.tiles_y = ((int64_t)h + BLUR_TH - 1) / BLUR_TH;
  p.k = (int32_t)k;
  const int K = (int)k;
  for (int i = 0; i < K; ++i)
    for (int j = 0; j < K; ++j)
      p.wts[i * K + j] = adjoint ? kernel[(K - 1 - i) * K + (K - 1 - j)] : kernel[i * K + j];
  const int64_t grid = (int64_t)nimg * p.tiles_x * p.tiles_y;
  if (grid > 0x7fffffffLL) return set_error(LIFTED_ETOOLARGE, "too many tiles");
  cudaError_t e;
  switch (K) {
    case 1: e = launch_blur<1>(p, grid, (cudaStream_t)stream); break;
    case 3: e = launch_blur<3>(p, grid, (cudaStream_t)stream); break;
    case 5: e = launch_blur<5>(p, grid, (cudaStream_t)stream); break;
    default: e = launch_blur<7>(p, grid, (cudaStream_t)stream); break;
  }
  if (e != cudaSuccess) return set_error(LIFTED_ECUDA, "blur launch: %s", cudaGetErrorString(e));
  count_launches(1);
  count_family(KF_BLUR, 1);
  return LIFTED_OK;
}

}  // extern "C"
