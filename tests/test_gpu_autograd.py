"""torch.autograd form: the backward is the adjoint lifting kernel (the
transform is linear, so the VJP is W^T g), checked by float64
finite-difference gradcheck and against the oracle's adjoint."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import autograd as ag  # noqa: E402


def test_gradcheck_db4_3d_crop():
    torch.manual_seed(0)
    x = torch.randn(32, 32, 32, dtype=torch.float64, device="cuda", requires_grad=True)
    f = lambda t: ag.dwt(t, "db4", "Zero", axes=(0, 1, 2), level=(2, 2, 2))  # noqa: E731
    assert torch.autograd.gradcheck(f, (x,), fast_mode=True, eps=1e-6, atol=1e-8)


def test_gradcheck_small_all_modes():
    torch.manual_seed(1)
    for mode in ("Zero", "Constant", "Periodic", "Symmetric", "Reflect"):
        x = torch.randn(6, 20, dtype=torch.float64, device="cuda", requires_grad=True)
        f = lambda t: ag.dwt(t, "cdf9.7", mode, axes=(1, 0), level=(2, 1))  # noqa: E731
        assert torch.autograd.gradcheck(f, (x,), eps=1e-6, atol=1e-8)
        g = lambda t: ag.idwt(t, "db3", mode, axes=(1,), level=(2,))  # noqa: E731
        assert torch.autograd.gradcheck(g, (x,), eps=1e-6, atol=1e-8)


def test_backward_is_reference_adjoint():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((32, 32, 32))
    gy = rng.standard_normal((32, 32, 32))
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    y = ag.dwt(xt, "db4", "Zero", axes=(0, 1, 2), level=(2, 2, 2))
    y.backward(torch.from_numpy(gy).cuda())
    rc, o = po.oracle_sep(gy, 4, 2, 0, [0, 1, 2], [2, 2, 2])
    assert rc == 0 and np.array_equal(xt.grad.cpu().numpy(), o)


def test_module_and_lsq_step_decreases_loss():
    torch.manual_seed(2)
    b = torch.randn(2, 64, 64, device="cuda")
    x = torch.zeros_like(b, requires_grad=True)
    W = ag.DWT("cdf9.7", "Zero", axes=(1, 2), level=(3, 3))
    opt = torch.optim.SGD([x], lr=0.5)
    losses = []
    for _ in range(5):
        opt.zero_grad()
        loss = 0.5 * torch.sum((x - b) ** 2) + 1e-3 * torch.sum(torch.abs(W(x)))
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < losses[0]
