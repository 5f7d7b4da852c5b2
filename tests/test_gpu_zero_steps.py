"""The Zero boundary's direct step code (zero_step in lw_line_kernel.cuh:
each update sums the taps inside the source band, in tap order) on the
general line kernel and the batch engine's whole and line items, bit for bit
against the oracle and against the exact step code it replaces (option
"zero_step_code" off): odd and ragged lengths (bands of ceil(m / 2) and
floor(m / 2) at every level), tiny bands at the deepest levels, where some
step's front and back edge ranges overlap and the host keeps the exact code,
contiguous and strided lines, every catalogue wavelet, all four transforms."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200 import pylifted as pl  # noqa: E402
from lifted_b200.batch import BatchPlan, lwt_images  # noqa: E402


def run(x, w, op, axes, levels):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    y = pl._lwt(t, w, 0, op, list(axes), list(levels), 1)
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.fixture
def exact_steps():
    def set_(on):
        _lib.set_option("zero_step_code", 0 if on else 1)
    yield set_
    _lib.set_option("zero_step_code", 1)


def levels_for(w, n):
    width = po.wavelet_width(w)
    return po.max_level(width, n) if width > 1 else max(1, int(np.log2(max(n, 2))))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_odd_lengths_every_wavelet(op, dtype, exact_steps):
    rng = np.random.default_rng(800 + op)
    cases = [((3, 1023), 1), ((1023, 5), 0), ((2, 4095), 1), ((777, 3), 0), ((6, 97), 1),
             ((33, 7), 0)]
    for w in po.wavelet_values():
        for shape, ax in cases:
            n = shape[ax]
            mx = levels_for(w, n)
            for lv in sorted({1, max(1, min(3, mx)), max(1, mx)}):
                x = rng.standard_normal(shape).astype(dtype)
                rc, o = po.oracle_sep(x, w, op, 0, [ax], [lv])
                if rc:
                    continue
                l0 = _lib.kernel_launches("line")
                g = run(x, w, op, [ax], [lv])
                assert np.array_equal(g, o), (w, shape, ax, lv)
                if _lib.kernel_launches("line") == l0:
                    continue  # served by another kernel
                exact_steps(True)
                try:
                    g2 = run(x, w, op, [ax], [lv])
                finally:
                    exact_steps(False)
                assert np.array_equal(g2, o), (w, shape, ax, lv)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_tiny_bands_and_levels_past_max(op):
    """Lengths 1..40 at every level count the oracle accepts (bands of one
    or two samples at the deepest levels)."""
    rng = np.random.default_rng(820 + op)
    for w in (2, 4, 100907, 5, 6, 10309):
        for n in range(1, 41):
            for lv in range(1, 6):
                x = rng.standard_normal((3, n)).astype(np.float32)
                rc, o = po.oracle_sep(x, w, op, 0, [1], [lv])
                if rc:
                    continue
                assert np.array_equal(run(x, w, op, [1], [lv]), o), (w, n, lv)
                xt = np.ascontiguousarray(x.T)
                rc, o = po.oracle_sep(xt, w, op, 0, [0], [lv])
                assert rc == 0
                assert np.array_equal(run(xt, w, op, [0], [lv]), o), (w, n, lv)


@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_odd_images_separable(op, exact_steps):
    """2D and 3D images with odd sides, both axes, CDF 9/7 and Daubechies4."""
    rng = np.random.default_rng(830 + op)
    for shape, axes, lv in [((1023, 1023), [0, 1], [4, 4]), ((255, 257), [0, 1], [3, 5]),
                            ((63, 65, 67), [0, 1, 2], [2, 3, 2])]:
        for w in (100907, 4):
            x = rng.standard_normal(shape).astype(np.float32)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            assert rc == 0
            assert np.array_equal(run(x, w, op, axes, lv), o), (shape, w)
            exact_steps(True)
            try:
                assert np.array_equal(run(x, w, op, axes, lv), o), (shape, w)
            finally:
                exact_steps(False)


@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_batch_whole_and_line_items(op, exact_steps):
    """Whole items of a 1D batch of short odd signals and line items of a
    persistent nD batch: both step codes give the oracle's result."""
    rng = np.random.default_rng(840 + op)
    lengths = [int(v) for v in rng.integers(64, 900, 40)]
    ws = [int(v) for v in rng.choice([2, 4, 100907, 5], 40)]
    lv = [max(1, min(5, levels_for(w, n))) for w, n in zip(ws, lengths)]
    x = rng.standard_normal(int(sum(lengths))).astype(np.float32)
    from test_batch_plan import oracle_batch
    want = oracle_batch(x, np.array(lengths), ws, lv, op, 0)
    shapes = [(int(a), int(b)) for a, b in rng.integers(40, 300, (12, 2))]
    iw = [int(v) for v in rng.choice([2, 4, 100907], 12)]
    ilv = [[max(1, min(3, levels_for(w, n))) for n in s] for s, w in zip(shapes, iw)]
    xs = [rng.standard_normal(s).astype(np.float32) for s in shapes]
    _lib.set_option("batch_nd_mode", 1)
    try:
        for exact in (False, True):
            exact_steps(exact)
            plan = BatchPlan(lengths, ws, lv, op=op, dtype="float32")
            y = plan.run(torch.from_numpy(x).cuda(), check=True)
            torch.cuda.synchronize()
            assert np.array_equal(y.cpu().numpy()[:len(x)], want), exact
            plan.close()
            ys = lwt_images([torch.from_numpy(a).cuda() for a in xs], iw, ilv, op=op)
            torch.cuda.synchronize()
            for a, b, w, l_ in zip(xs, ys, iw, ilv):
                rc, o = po.oracle_sep(a, w, op, 0, [0, 1], l_)
                assert rc == 0
                assert np.array_equal(b.cpu().numpy(), o), (a.shape, w, l_, exact)
    finally:
        _lib.set_option("batch_nd_mode", 0)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0
