"""Strided passes over lines of any length on the TMA-staged kernel (Zero
boundary): at a level whose input band has odd length m the s band holds
ceil(m / 2) values and the d band floor(m / 2), so the end-masked
instantiation masks taps by the source band's own length, stores s and d
up to their own ends, and reads each detail band from ceil(n / 2^l).  Whole
lines, 512-sample windows with halos, a chained band launch, 3D views;
compiled and generic wavelets; bit for bit against the oracle, and no pass
on the general kernel."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200 import pylifted as pl  # noqa: E402

CASES = [((1023, 64), 3), ((4095, 64), 6), ((777, 96), 4), ((511, 32), 5), ((33, 64), 2),
         ((255, 4, 64), 4), ((1081, 48), 3), ((4064, 32), 6), ((3, 64), 1)]


def run(x, w, op, axes, levels, fams=("col",)):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    l0 = _lib.kernel_launches("line")
    c0 = sum(_lib.kernel_launches(f) for f in fams)
    y = pl._lwt(t, w, 0, op, list(axes), list(levels), 1)
    torch.cuda.synchronize()
    return (y.cpu().numpy(), _lib.kernel_launches("line") - l0,
            sum(_lib.kernel_launches(f) for f in fams) - c0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_odd_strided_lines_on_the_tma_kernel(op, dtype):
    rng = np.random.default_rng(900 + op)
    for w in (2, 4, 100907, 5, 104):
        width = po.wavelet_width(w)
        for shape, lv in CASES:
            lv = max(1, min(lv, po.max_level(width, shape[0])))
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, [0], [lv])
            if rc:
                continue
            g, general, col = run(x, w, op, [0], [lv])
            assert np.array_equal(g, o), (w, shape, lv, np.argwhere(g != o)[:4])
            # bands long enough that no step's edge ranges overlap run fast
            if shape[0] >= 255:
                assert general == 0 and col > 0, (w, shape, lv, general, col)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_every_catalogue_wavelet_odd_columns(op):
    rng = np.random.default_rng(920 + op)
    for w in po.wavelet_values():
        width = po.wavelet_width(w)
        for shape in ((1023, 32), (4095, 32)):
            mx = po.max_level(width, shape[0]) if width > 1 else 8
            for lv in sorted({1, max(1, min(4, mx)), max(1, mx)}):
                x = rng.standard_normal(shape).astype(np.float32)
                rc, o = po.oracle_sep(x, w, op, 0, [0], [lv])
                if rc:
                    continue
                g, _, _ = run(x, w, op, [0], [lv])
                assert np.array_equal(g, o), (w, shape, lv)


@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_odd_image_axis0(op):
    """4095 x 4096 float32 CDF 9/7, 6 levels on axis 0: one window launch and
    one band launch of the TMA-staged kernel."""
    rng = np.random.default_rng(940 + op)
    x = rng.standard_normal((4095, 4096)).astype(np.float32)
    rc, o = po.oracle_sep(x, 100907, op, 0, [0], [6])
    assert rc == 0
    g, general, col = run(x, 100907, op, [0], [6])
    assert np.array_equal(g, o)
    assert general == 0 and col == 2, (general, col)


UNALIGNED = [((4095, 4095), [0], [6]), ((1023, 1023), [0], [4]), ((777, 99), [0], [4]),
             ((127, 63, 99), [0], [3]), ((127, 63, 99), [1], [3]), ((500, 31), [0], [5]),
             ((300, 5, 7), [0], [3]), ((1024, 1023), [0], [6])]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_unaligned_strides_plain_load_staging(op, dtype):
    """Strides, line counts or slice strides that are not multiples of 16
    bytes (odd-width images, 3D views with odd inner extents, fewer than 32
    lines): the plain-load instantiation stages the tiles; every pass bit
    for bit against the oracle and none on the general kernel."""
    rng = np.random.default_rng(960 + op)
    for w in (2, 4, 100907, 5, 104):
        width = po.wavelet_width(w)
        for shape, axes, lv in UNALIGNED:
            lv = [max(1, min(l_, po.max_level(width, shape[a]))) for a, l_ in zip(axes, lv)]
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            if rc:
                continue
            # (the register tile kernel takes strided lines of a multiple of
            # 32 samples before the plain-load form)
            g, general, col = run(x, w, op, axes, lv, ("col", "reg"))
            assert np.array_equal(g, o), (w, shape, axes, lv, np.argwhere(g != o)[:4])
            # float64 whole lines of more levels than its registers hold need
            # a band a multiple of 32 long for the next launch
            if dtype == np.float32:
                assert general == 0 and col > 0, (w, shape, axes, lv, general, col)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


def test_unaligned_strides_other_boundaries_stay_exact():
    rng = np.random.default_rng(980)
    x = rng.standard_normal((1023, 1023)).astype(np.float32)
    for bc in (1, 2, 3, 4):
        for op in range(4):
            rc, o = po.oracle_sep(x, 100907, op, bc, [0], [3])
            assert rc == 0
            t = torch.from_numpy(x).cuda()
            y = pl._lwt(t, 100907, bc, op, [0], [3], 1)
            assert np.array_equal(y.cpu().numpy(), o), (bc, op)
