"""Wavelet-regularised least squares through the differentiable DWT.

    loss(x) = 0.5 * ||A x - b||^2 + lam * ||W x||_1

with A a fixed 5 x 5 blur (zero padding, 'same' size, applied per image) and
W the separable lifting DWT over the last two axes.  Gradient descent runs
through ``lifted_b200.autograd``: the backward of W is the ForwardAdjoint
lifting kernel, so d/dx lam * ||W x||_1 = lam * W^T sign(W x) comes from the
adjoint kernel, not from saved activations.

``make_problem`` builds the seeded synthetic problem (piecewise-constant
ground truth of random rectangles, b = A x_true + noise); ``GradientLoop``
runs the steps on the GPU; the float64 CPU check of the same iteration lives
in the tests (it uses the oracle).

A is applied by the library's own float32 correlation kernel
(``lifted_blur2d_f32``), forward and adjoint, so the gradient of the data
term carries no TF32 rounding.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import autograd as ag


def blur_kernel(seed: int, size: int = 5) -> np.ndarray:
    """Seeded positive 5 x 5 kernel normalised to sum 1."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(0.1, 1.0, (size, size))
    return k / k.sum()


def make_problem(batch: int, n: int, seed: int = 1005, rects: int = 64,
                 noise_var: float = 0.01):
    """x_true (batch, n, n): `rects` random axis-aligned rectangles with
    N(0, 1) levels per image; b = A x_true + N(0, noise_var).  Returns
    float64 numpy arrays (x_true, b, kernel)."""
    rng = np.random.default_rng(seed)
    k = blur_kernel(seed + 1)
    xt = np.zeros((batch, n, n))
    for i in range(batch):
        for _ in range(rects):
            y0, x0 = rng.integers(0, n, 2)
            h, w = rng.integers(n // 64 + 1, n // 4 + 2, 2)
            xt[i, y0:y0 + h, x0:x0 + w] = rng.standard_normal()
    b = blur_np(xt, k) + rng.normal(0.0, np.sqrt(noise_var), xt.shape)
    return xt, b, k


def blur_np(x: np.ndarray, k: np.ndarray) -> np.ndarray:
    """A x: 2-D correlation with k, zero padding, 'same' size (float64)."""
    r = k.shape[0] // 2
    n0, n1 = x.shape[-2:]
    xp = np.zeros(x.shape[:-2] + (n0 + 2 * r, n1 + 2 * r))
    xp[..., r:r + n0, r:r + n1] = x
    out = np.zeros_like(x, dtype=np.float64)
    for i in range(k.shape[0]):
        for j in range(k.shape[1]):
            out += k[i, j] * xp[..., i:i + n0, j:j + n1]
    return out


def blur_adj_np(y: np.ndarray, k: np.ndarray) -> np.ndarray:
    """A^T y: correlation with the flipped kernel (zero padding)."""
    return blur_np(y, k[::-1, ::-1])


def blur2d(x, kernel: np.ndarray, adjoint: bool = False):
    """A x (or A^T x) for a float32 CUDA tensor (..., h, w): correlation of
    each image with `kernel` (odd size <= 7), zero padding, same size."""
    import torch

    if x.dtype != torch.float32 or not x.is_cuda:
        raise TypeError("blur2d takes a float32 CUDA tensor")
    x = x.contiguous()
    out = torch.empty_like(x)
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    h, w = x.shape[-2], x.shape[-1]
    nimg = x.numel() // max(h * w, 1)
    lib = _lib.load()
    stream = torch.cuda.current_stream(x.device).cuda_stream
    _lib.check(lib.lifted_blur2d_f32(x.data_ptr(), out.data_ptr(), nimg, h, w,
                                     k.ctypes.data_as(ctypes.c_void_p), k.shape[0],
                                     1 if adjoint else 0, stream))
    return out


def _blur_function():
    import torch

    class Blur(torch.autograd.Function):
        """A as an autograd Function: backward is A^T (the flipped kernel)."""

        @staticmethod
        def forward(ctx, x, kernel):
            ctx.kernel = kernel
            return blur2d(x, kernel)

        @staticmethod
        def backward(ctx, g):
            return blur2d(g, ctx.kernel, adjoint=True), None

    return Blur


class GradientLoop:
    """Gradient descent on the loss above, float32 on one CUDA device."""

    def __init__(self, b, kernel, lam: float, step: float, wavelet="cdf9.7",
                 levels=(5, 5), device="cuda"):
        import torch

        self.torch = torch
        self.b = torch.as_tensor(b, dtype=torch.float32, device=device)
        self.kernel = np.ascontiguousarray(kernel, dtype=np.float32)
        self._blur = _blur_function()
        self.lam, self.step_size = float(lam), float(step)
        nd = self.b.ndim
        self.W = ag.DWT(wavelet, "Zero", axes=(nd - 2, nd - 1), level=tuple(levels))
        self.x = torch.zeros_like(self.b, requires_grad=True)

    def blur(self, x):
        return self._blur.apply(x, self.kernel)

    def loss(self, x):
        r = self.blur(x) - self.b
        return 0.5 * (r * r).sum() + self.lam * self.W(x).abs().sum()

    def step(self):
        """One gradient step; returns the loss before the step (a CUDA
        scalar tensor, not synchronised)."""
        torch = self.torch
        self.x.grad = None
        f = self.loss(self.x)
        f.backward()
        with torch.no_grad():
            self.x -= self.step_size * self.x.grad
        return f.detach()
