"""The generic register kernels (one instantiation for every catalogue
wavelet, each step dispatched at run time on its compiled shape) against the
oracle, bit for bit: all 34 catalogue wavelets, all four transforms,
float32 and float64, on the row lengths the warp-per-row kernel takes and
every level count the wavelet's reach allows there; and against the general
line kernel they replace (option off)."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200 import pylifted as pl  # noqa: E402


def run(x, w, op, axes, levels):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    n0 = _lib.launch_count()
    y = pl._lwt(t, w, 0, op, list(axes), list(levels), 1)
    torch.cuda.synchronize()
    return y.cpu().numpy(), _lib.launch_count() - n0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_all_catalogue_wavelets_on_rows(op, dtype):
    rng = np.random.default_rng(90 + op)
    for w in po.wavelet_values():
        width = po.wavelet_width(w)
        for n in (512, 2048):
            mx = po.max_level(width, n) if width > 1 else int(np.log2(n))
            for lv in sorted({1, 2, min(3, mx), mx}):
                if lv < 1:
                    continue
                x = rng.standard_normal((5, n)).astype(dtype)
                rc, o = po.oracle_sep(x, w, op, 0, [1], [lv])
                if rc:
                    continue
                g, _ = run(x, w, op, [1], [lv])
                assert np.array_equal(g, o), (w, n, lv)
                _lib.set_option("generic_kernels", 0)
                try:
                    g2, _ = run(x, w, op, [1], [lv])
                finally:
                    _lib.set_option("generic_kernels", 1)
                assert np.array_equal(g2, o), (w, n, lv)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_all_catalogue_wavelets_strided(op, dtype):
    """Strided lines on the generic TMA-staged kernel: whole columns, long
    columns on windows plus a band launch, short lines of a 3D view stacked
    per window, and a 2D separable transform; every catalogue wavelet."""
    rng = np.random.default_rng(95 + op)
    cases = [((512, 64), [0]), ((2048, 64), [0]), ((64, 8, 64), [0]), ((256, 96), [0, 1]),
             ((8192, 32), [0])]
    for w in po.wavelet_values():
        width = po.wavelet_width(w)
        for shape, axes in cases:
            lv = []
            for a in axes:
                n = shape[a]
                mx = po.max_level(width, n) if width > 1 else int(np.log2(n))
                lv.append(max(1, min(6 if n > 4096 else 4, mx)))
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            if rc:
                continue
            g, _ = run(x, w, op, axes, lv)
            assert np.array_equal(g, o), (w, shape, axes, lv)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_all_catalogue_wavelets_long_rows(op, dtype):
    """Rows longer than one warp holds on the generic windowed kernel (first,
    last and shorter windows clipped by the row): every catalogue wavelet."""
    rng = np.random.default_rng(99 + op)
    for w in po.wavelet_values():
        width = po.wavelet_width(w)
        n = 12288
        mx = po.max_level(width, n) if width > 1 else int(np.log2(n))
        for lv in sorted({1, max(1, min(3, mx))}):
            x = rng.standard_normal((2, n)).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, [1], [lv])
            if rc:
                continue
            g, _ = run(x, w, op, [1], [lv])
            assert np.array_equal(g, o), (w, n, lv)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_rows_of_other_lengths_on_windows(op, dtype):
    """Row lengths that are multiples of 2^levels but not of a lane's pairs
    (1000, 1080, 1920, 3000, 12000 samples): the band ends inside a lane, the
    windowed kernel masks it; compiled and generic wavelets, bit for bit."""
    rng = np.random.default_rng(120 + op)
    for w in (2, 4, 100907, 5, 104, 17):
        width = po.wavelet_width(w)
        for n in (1000, 1080, 1920, 3000, 12000):
            tz = (n & -n).bit_length() - 1  # levels that keep every band even
            mx = po.max_level(width, n) if width > 1 else int(np.log2(n))
            for lv in sorted({1, min(tz, mx, 3)}):
                if lv < 1:
                    continue
                x = rng.standard_normal((3, n)).astype(dtype)
                rc, o = po.oracle_sep(x, w, op, 0, [1], [lv])
                if rc:
                    continue
                g, _ = run(x, w, op, [1], [lv])
                assert np.array_equal(g, o), (w, n, lv)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_columns_and_images_of_other_lengths(op, dtype):
    """Strided lines whose length is a multiple of 2^levels but not of 32
    (whole lines, windows, a chained band, 3D views) and 2D images of such
    sizes (1080 x 1920, 1000 x 3000): compiled and generic wavelets, bit for
    bit against the oracle."""
    rng = np.random.default_rng(130 + op)
    cases = [((200, 64), [0], [3]), ((1000, 64), [0], [3]), ((1080, 96), [0], [3]),
             ((1920, 32), [0], [6]), ((3000, 32), [0], [3]), ((1000, 4, 32), [0], [3]),
             ((16, 8, 64), [1], [1]), ((48, 6, 32), [0, 1], [4, 1]),
             ((1080, 1920), [0, 1], [3, 3]), ((1000, 3000), [0, 1], [3, 2])]
    for w in (2, 4, 100907, 5, 104):
        for shape, axes, lv in cases:
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            if rc:
                continue
            g, _ = run(x, w, op, axes, lv)
            assert np.array_equal(g, o), (w, shape, axes, lv)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_columns_of_partial_line_groups(op, dtype):
    """Strided passes whose line count is not a multiple of 32 (the last
    group of 32 lines is partial): 2D columns, 3D views with an outer dim,
    whole lines, windows and a chained band pass (the band buffer's boxes
    start at outer * lines + first line), bit for bit against the oracle."""
    rng = np.random.default_rng(170 + op)
    cases = [((512, 100), [0], [4]), ((1000, 3000), [0], [3]), ((200, 36), [0], [3]),
             ((64, 6, 36), [0], [2]), ((4, 600, 36), [1], [3]), ((4, 2048, 36), [1], [6]),
             ((3, 256, 100), [1], [5])]
    for w in (2, 4, 33, 100907, 5):
        for shape, axes, lv in cases:
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            if rc:
                continue
            g, _ = run(x, w, op, axes, lv)
            assert np.array_equal(g, o), (w, shape, axes, lv)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_float64_strided_passes_take_the_same_kernels_as_float32(op):
    """Every catalogue wavelet's strided pass, the wide-reach ones (reach
    6-9, single-buffered mailbox in float64) included: float64 falls back to
    the general line kernel exactly where float32 does, and both are bit for
    bit equal to the oracle."""
    rng = np.random.default_rng(180 + op)
    shape = (2048, 64)
    for w in po.wavelet_values():
        width = po.wavelet_width(w)
        mx = po.max_level(width, shape[0]) if width > 1 else int(np.log2(shape[0]))
        lv = max(1, min(4, mx))
        general = {}
        for dtype in (np.float32, np.float64):
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, [0], [lv])
            if rc:
                break
            l0 = _lib.kernel_launches("line")
            g, _ = run(x, w, op, [0], [lv])
            general[dtype] = _lib.kernel_launches("line") - l0
            assert np.array_equal(g, o), (w, dtype, lv)
        else:
            assert general[np.float64] == general[np.float32], (w, lv, general)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0
