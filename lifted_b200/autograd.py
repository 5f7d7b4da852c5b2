"""Differentiable lifting DWT for PyTorch.

The transform is linear, so the vector-Jacobian product of y = W x is
W^T g: the backward of the forward transform is the ForwardAdjoint lifting
kernel on the incoming gradient, and the backward of the inverse transform
is the InverseAdjoint kernel.  No activations are saved.

    y = lifted_b200.autograd.dwt(x, "cdf9.7", mode="Zero", axes=(1, 2),
                                 level=(5, 5))
    y.backward(g)          # x.grad = W^T g, by the adjoint kernel
"""
from __future__ import annotations

import torch

from . import pylifted as _pl


def _run(op, x, wavelet, mode, axes, level):
    return _pl._lwt(x, wavelet, mode, op, axes, level, 1)


class LiftedDWT(torch.autograd.Function):
    """y = W x (Forward); dL/dx = W^T dL/dy (ForwardAdjoint)."""

    @staticmethod
    def forward(ctx, x, wavelet, mode, axes, level):
        ctx.cfg = (wavelet, mode, axes, level)
        return _run(_pl.Transform.Forward, x, wavelet, mode, axes, level)

    @staticmethod
    def backward(ctx, g):
        wavelet, mode, axes, level = ctx.cfg
        gx = _run(_pl.Transform.ForwardAdjoint, g, wavelet, mode, axes, level)
        return gx, None, None, None, None


class LiftedIDWT(torch.autograd.Function):
    """x = W^{-1} y (Inverse); dL/dy = W^{-T} dL/dx (InverseAdjoint)."""

    @staticmethod
    def forward(ctx, y, wavelet, mode, axes, level):
        ctx.cfg = (wavelet, mode, axes, level)
        return _run(_pl.Transform.Inverse, y, wavelet, mode, axes, level)

    @staticmethod
    def backward(ctx, g):
        wavelet, mode, axes, level = ctx.cfg
        gy = _run(_pl.Transform.InverseAdjoint, g, wavelet, mode, axes, level)
        return gy, None, None, None, None


def _norm(axes, level):
    axes = tuple(axes) if axes is not None and not isinstance(axes, int) else axes
    level = tuple(level) if not isinstance(level, int) else level
    return axes, level


def dwt(x, wavelet, mode=_pl.BoundaryCondition.Zero, axes=None, level=1):
    """Differentiable forward transform (see pylifted.lwt_forward)."""
    axes, level = _norm(axes, level)
    return LiftedDWT.apply(x, wavelet, mode, axes, level)


def idwt(y, wavelet, mode=_pl.BoundaryCondition.Zero, axes=None, level=1):
    """Differentiable inverse transform (see pylifted.lwt_inverse)."""
    axes, level = _norm(axes, level)
    return LiftedIDWT.apply(y, wavelet, mode, axes, level)


class DWT(torch.nn.Module):
    """Module form of dwt()."""

    def __init__(self, wavelet, mode=_pl.BoundaryCondition.Zero, axes=None, level=1):
        super().__init__()
        self.wavelet, self.mode = wavelet, mode
        self.axes, self.level = _norm(axes, level)

    def forward(self, x):
        return LiftedDWT.apply(x, self.wavelet, self.mode, self.axes, self.level)
