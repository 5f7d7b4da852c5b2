"""Full-size checks of the benchmark configurations on the GPU, through the
C ABI: exact agreement with the CPU oracle where it finishes in seconds,
and size-independent properties (inverse round trip, the adjoint
dot-product identity <W x, y> = <x, W^T y>) at full size."""
import numpy as np
import pytest

import pyoracle as po
from helpers import f32_bound

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import pylifted as pl  # noqa: E402


def cfg2_image(seed=1002, n=4096):
    """32 Gaussian blobs + N(0, 0.01) noise (variance 0.01), float32."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float32)
    img = np.zeros((n, n), np.float32)
    for _ in range(32):
        cy, cx = rng.uniform(0, n, 2)
        sig = rng.uniform(16, 256)
        amp = rng.standard_normal()
        img += amp * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * sig * sig)).astype(np.float32)
    img += rng.normal(0, 0.1, (n, n)).astype(np.float32)
    return img


def test_cfg1_db2_f64_exact_roundtrip_and_adjoint():
    rng = np.random.default_rng(1001)
    x = rng.standard_normal((64, 65536))
    v = rng.standard_normal((64, 65536))
    xt = torch.from_numpy(x).cuda()
    vt = torch.from_numpy(v).cuda()
    wx = pl.lwt_forward(xt, "db2", "Zero", axes=(1,), level=(5,))
    rc, o = po.oracle_sep(x, 2, 0, 0, [1], [5])
    assert rc == 0 and np.array_equal(wx.cpu().numpy(), o)
    back = pl.lwt_inverse(wx, "db2", "Zero", axes=(1,), level=(5,))
    assert torch.max(torch.abs(back - xt)).item() <= 1e-13 * torch.max(torch.abs(xt)).item() * 10
    wtv = pl.lwt_forward_adjoint(vt, "db2", "Zero", axes=(1,), level=(5,))
    rc, oa = po.oracle_sep(v, 2, 2, 0, [1], [5])
    assert rc == 0 and np.array_equal(wtv.cpu().numpy(), oa)
    a = torch.sum(vt * wx).item()
    b = torch.sum(wtv * xt).item()
    assert abs(a - b) <= 1e-12 * max(abs(a), abs(b))
    for bc in range(1, 5):
        wx = pl.lwt_forward(xt, "db2", bc, axes=(1,), level=(5,))
        rc, o = po.oracle_sep(x, 2, 0, bc, [1], [5])
        assert rc == 0 and np.array_equal(wx.cpu().numpy(), o), bc


def test_cfg2_cdf97_f32_fwd_adjoint_vs_oracle():
    x = cfg2_image()
    xt = torch.from_numpy(x).cuda()
    w = pl.lwt_forward(xt, "cdf9.7", "Zero", axes=(0, 1), level=(6, 6))
    a = pl.lwt_forward_adjoint(w, "cdf9.7", "Zero", axes=(0, 1), level=(6, 6))
    rc, ow = po.oracle_sep(x, 100907, 0, 0, [0, 1], [6, 6])
    assert rc == 0
    wn = w.cpu().numpy()
    assert np.max(np.abs(wn - ow)) <= f32_bound(ow)
    assert np.array_equal(wn, ow)
    rc, oa = po.oracle_sep(ow, 100907, 2, 0, [0, 1], [6, 6])
    an = a.cpu().numpy()
    assert rc == 0 and np.array_equal(an, oa)
    # float64 dot-product identity at full size
    x64 = torch.from_numpy(x.astype(np.float64)).cuda()
    y64 = torch.randn_like(x64)
    wx = pl.lwt_forward(x64, "cdf9.7", "Zero", axes=(0, 1), level=(6, 6))
    wty = pl.lwt_forward_adjoint(y64, "cdf9.7", "Zero", axes=(0, 1), level=(6, 6))
    p, q = torch.sum(y64 * wx).item(), torch.sum(wty * x64).item()
    assert abs(p - q) <= 1e-12 * max(abs(p), abs(q))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_cfg3_db4_3d_roundtrip(dtype):
    rng = np.random.default_rng(1003)
    n = 128
    x = rng.standard_normal((n, n, n)).astype(dtype)
    xt = torch.from_numpy(x).cuda()
    w = pl.lwt_forward(xt, "db4", "Zero", axes=(0, 1, 2), level=(4, 4, 4))
    back = pl.lwt_inverse(w, "db4", "Zero", axes=(0, 1, 2), level=(4, 4, 4))
    tol = 1e-12 if dtype == np.float64 else 1e-4
    assert torch.max(torch.abs(back - xt)).item() <= tol * torch.max(torch.abs(xt)).item()
    rc, o = po.oracle_sep(x, 4, 0, 0, [0, 1, 2], [4, 4, 4])
    assert rc == 0 and np.array_equal(w.cpu().numpy(), o)
