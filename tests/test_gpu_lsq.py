"""Wavelet-regularised least squares through the autograd DWT (float32 on
the GPU) against the same gradient iteration in float64 on the CPU with the
oracle's Forward and ForwardAdjoint: the loss trajectories agree to float32
accuracy and the loss decreases."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import lsq  # noqa: E402


def cpu_losses(b, k, lam, eta, steps, levels):
    losses = []
    for i in range(b.shape[0]):
        x = np.zeros_like(b[i])
        li = []
        for _ in range(steps):
            r = lsq.blur_np(x, k) - b[i]
            rc, wx = po.oracle_sep(x, 100907, 0, 0, [0, 1], list(levels))
            assert rc == 0
            li.append(0.5 * float(np.sum(r * r)) + lam * float(np.sum(np.abs(wx))))
            rc, wts = po.oracle_sep(np.sign(wx), 100907, 2, 0, [0, 1], list(levels))
            assert rc == 0
            x = x - eta * (lsq.blur_adj_np(r, k) + lam * wts)
        losses.append(li)
    return np.sum(np.array(losses), axis=0)


def test_lsq_matches_fp64_cpu_iteration():
    lam, eta, steps, levels = 0.02, 1.0, 12, (4, 4)
    xt, b, k = lsq.make_problem(2, 256, seed=7, rects=16)
    loop = lsq.GradientLoop(b, k, lam, eta, levels=levels)
    g = np.array([float(loop.step()) for _ in range(steps)])
    c = cpu_losses(b, k, lam, eta, steps, levels)
    rel = np.abs(g - c) / np.abs(c)
    assert rel.max() < 1e-4, rel
    assert g[-1] < 0.5 * g[0]


def test_blur_adjoint_is_transpose():
    rng = np.random.default_rng(3)
    k = lsq.blur_kernel(3)
    x = rng.standard_normal((2, 40, 33))
    y = rng.standard_normal((2, 40, 33))
    lhs = np.sum(lsq.blur_np(x, k) * y)
    rhs = np.sum(x * lsq.blur_adj_np(y, k))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
