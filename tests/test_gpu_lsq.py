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


@pytest.mark.parametrize("ksize", [3, 5, 7])
def test_blur_kernel_matches_float64(ksize):
    """The library's blur (A and A^T) against the float64 numpy reference:
    float32 accumulation of at most 49 products, tolerance 1e-6 of the
    image scale; sizes that leave partial tiles."""
    rng = np.random.default_rng(11 + ksize)
    k = rng.uniform(0.1, 1.0, (ksize, ksize))
    k /= k.sum()
    for shape in [(3, 100, 77), (1, 2048, 64), (2, 33, 130)]:
        x = rng.standard_normal(shape).astype(np.float32)
        xt = torch.from_numpy(x).cuda()
        for adj, ref in ((False, lsq.blur_np), (True, lsq.blur_adj_np)):
            got = lsq.blur2d(xt, k, adjoint=adj).cpu().numpy()
            want = ref(x.astype(np.float64), k.astype(np.float32).astype(np.float64))
            assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want)) * ksize, (shape, adj)


def test_blur_abi_checks():
    import ctypes
    from lifted_b200 import _lib

    lib = _lib.load()
    x = torch.zeros(1, 16, 16, device="cuda")
    y = torch.zeros_like(x)
    k = np.ones((4, 4), dtype=np.float32)
    s = torch.cuda.current_stream().cuda_stream
    kp = k.ctypes.data_as(ctypes.c_void_p)
    assert lib.lifted_blur2d_f32(x.data_ptr(), y.data_ptr(), 1, 16, 16, kp, 4, 0, s) == _lib.EINVAL
    h = np.zeros(256, dtype=np.float32)
    assert lib.lifted_blur2d_f32(h.ctypes.data, y.data_ptr(), 1, 16, 16, kp, 3, 0, s) == _lib.EINVAL
    assert lib.lifted_blur2d_f32(x.data_ptr(), x.data_ptr(), 1, 16, 16, kp, 3, 0, s) == _lib.EINVAL
