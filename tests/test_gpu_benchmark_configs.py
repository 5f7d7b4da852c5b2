"""Parity on the benchmark configurations themselves, bit for bit against the
oracle:

* the 3D volume: 512^3 Daubechies4, levels (4, 4, 4) on axes (0, 1, 2),
  through the torch.autograd.Function (forward = Forward, backward =
  ForwardAdjoint of the incoming gradient), float32 at full size and float64
  on two 512 x 512 x 64 slabs that drive the same kernels (512-sample rows
  whose fourth level runs on compacted lanes; 512-line strided passes; the
  64-sample strided lines of the other slab stacked per window);
* the batched uneven 1D form over the benchmark's full length range
  (round(2^U[8, 20]) samples, every catalogue wavelet, levels
  U{1..max_level}), Forward and ForwardAdjoint through one persistent
  launch each.

The reference's separable driver (src/lifted-drivers-inl.hpp:417-486) is
what the oracle restates."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200 import autograd as ag  # noqa: E402
from lifted_b200.batch import BatchPlan  # noqa: E402
from test_batch_plan import oracle_batch  # noqa: E402

DB4 = 4


def smoothed_volume(shape, seed, dtype):
    """N(0,1) smoothed by an edge-clamped 3-point box along every axis."""
    v = np.random.default_rng(seed).standard_normal(shape)
    for ax in range(len(shape)):
        n = shape[ax]
        p = np.concatenate([np.take(v, [0], ax), v, np.take(v, [n - 1], ax)], axis=ax)
        v = (np.take(p, range(0, n), ax) + np.take(p, range(1, n + 1), ax) +
             np.take(p, range(2, n + 2), ax)) / 3
    return np.ascontiguousarray(v.astype(dtype))


def forward_and_backward(x, levels):
    """y = W x and x.grad = W^T y through the autograd Function."""
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    y = ag.dwt(xt, "db4", "Zero", axes=(0, 1, 2), level=levels)
    y.backward(y.detach())
    torch.cuda.synchronize()
    return y.detach().cpu().numpy(), xt.grad.cpu().numpy()


def check_volume(x, levels):
    c0 = _lib.kernel_launches("col")
    l0 = _lib.kernel_launches("line")
    y, gx = forward_and_backward(x, levels)
    assert _lib.kernel_launches("col") > c0, "strided passes missed the TMA-staged kernel"
    assert _lib.kernel_launches("line") == l0, "a pass fell back to the general kernel"
    rc, oy = po.oracle_sep(x, DB4, 0, 0, [0, 1, 2], list(levels))
    assert rc == 0
    assert np.array_equal(y, oy), np.argwhere(y != oy)[:5]
    rc, og = po.oracle_sep(oy, DB4, 2, 0, [0, 1, 2], list(levels))
    assert rc == 0
    assert np.array_equal(gx, og), np.argwhere(gx != og)[:5]


def test_volume_512_cubed_float32():
    check_volume(smoothed_volume((512, 512, 512), 1003, np.float32), (4, 4, 4))


@pytest.mark.parametrize("shape", [(64, 512, 512), (512, 512, 64)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_volume_slabs(shape, dtype):
    check_volume(smoothed_volume(shape, 1013, dtype), (4, 4, 4))


@pytest.mark.parametrize("op", [0, 2])
def test_batch_full_length_range(op):
    rng = np.random.default_rng(1014 + op)
    n = 300
    lengths = np.round(2.0 ** rng.uniform(8, 20, n)).astype(np.int64)
    allw = po.wavelet_values()
    ws = [allw[i] for i in rng.integers(0, len(allw), n)]
    lv = []
    for L, w in zip(lengths, ws):
        width = po.wavelet_width(w)
        mx = int(np.floor(np.log2(L))) if width == 1 else po.max_level(width, int(L))
        lv.append(int(rng.integers(1, max(mx, 1) + 1)))
    x = rng.standard_normal(int(lengths.sum())).astype(np.float32)
    want = oracle_batch(x, lengths, ws, lv, op, 0)
    plan = BatchPlan(lengths, ws, lv, op=op, dtype="float32")
    assert plan.info["ntiles"] > 0 and plan.info["nwhole"] > 0
    b0 = _lib.kernel_launches("batch")
    xt = torch.from_numpy(x).cuda()
    got = plan.run(xt, graph=True, check=True)
    torch.cuda.synchronize()
    assert _lib.kernel_launches("batch") == b0 + 1, "one persistent launch per transform"
    got = got.cpu().numpy()[:len(x)]
    assert np.array_equal(got, want), np.argwhere(got != want)[:5]
    plan.close()
