"""The register-blocked fast path (whole-line contiguous, whole-line strided
and tiled strided launches) against the CPU oracle, bit for bit, and against
the general line kernel (fast path switched off), on shapes that select it:
lengths that are multiples of the chunk size, Zero boundary, the compiled
wavelets (Daubechies2, Daubechies4, CDF9_7), all four transforms."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200 import pylifted as pl  # noqa: E402

WAVELETS = [2, 4, 100907]


@pytest.fixture(autouse=True)
def fast_on():
    _lib.set_option("fast_path", 1)
    yield
    _lib.set_option("fast_path", 1)


def run(x, w, tf, bc, axes, levels, fast=True):
    _lib.set_option("fast_path", 1 if fast else 0)
    try:
        t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        n0 = _lib.launch_count()
        y = pl._lwt(t, w, bc, tf, list(axes), list(levels), 1)
        torch.cuda.synchronize()
        return y.cpu().numpy(), _lib.launch_count() - n0
    finally:
        _lib.set_option("fast_path", 1)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rows_whole_line(dtype):
    rng = np.random.default_rng(21)
    for w in WAVELETS:
        for n in (32, 64, 256, 512, 1024, 2048, 4096):
            for lv in (1, 2, 3, 4, 5, 6, 9):
                x = rng.standard_normal((3, n)).astype(dtype)
                for tf in range(4):
                    rc, o = po.oracle_sep(x, w, tf, 0, [1], [lv])
                    if rc:
                        continue
                    g, _ = run(x, w, tf, 0, [1], [lv])
                    assert np.array_equal(g, o), (dtype, w, n, lv, tf)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_columns_whole_and_tiled(dtype):
    rng = np.random.default_rng(22)
    for w in WAVELETS:
        for n in (64, 256, 512, 1024, 2048):
            for lv in (1, 3, 4, 6):
                x = rng.standard_normal((n, 40 if (lv + n) % 2 else 41)).astype(dtype)
                for tf in range(4):
                    rc, o = po.oracle_sep(x, w, tf, 0, [0], [lv])
                    if rc:
                        continue
                    g, _ = run(x, w, tf, 0, [0], [lv])
                    assert np.array_equal(g, o), (dtype, w, n, lv, tf)


def test_2d_cdf97_like_headline():
    rng = np.random.default_rng(23)
    x = rng.standard_normal((1024, 512)).astype(np.float32)
    for tf in range(4):
        rc, o = po.oracle_sep(x, 100907, tf, 0, [0, 1], [6, 6])
        assert rc == 0
        g, launches = run(x, 100907, tf, 0, [0, 1], [6, 6])
        assert np.array_equal(g, o), tf
        g2, _ = run(x, 100907, tf, 0, [0, 1], [6, 6], fast=False)
        assert np.array_equal(g, g2)


def test_3d_db4_fast_path():
    rng = np.random.default_rng(24)
    for dtype in (np.float32, np.float64):
        x = rng.standard_normal((64, 32, 128)).astype(dtype)
        for tf in (0, 2):
            rc, o = po.oracle_sep(x, 4, tf, 0, [0, 1, 2], [3, 2, 4])
            g, _ = run(x, 4, tf, 0, [0, 1, 2], [3, 2, 4])
            assert rc == 0 and np.array_equal(g, o), (dtype, tf)


def test_other_boundaries_fall_back_exactly():
    rng = np.random.default_rng(25)
    x = rng.standard_normal((64, 256)).astype(np.float32)
    for bc in (1, 2, 3, 4):
        for tf in (0, 2):
            rc, o = po.oracle_sep(x, 100907, tf, bc, [1, 0], [4, 3])
            g, _ = run(x, 100907, tf, bc, [1, 0], [4, 3])
            assert rc == 0 and np.array_equal(g, o), (bc, tf)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_tma_strided_windows_and_whole_lines(op, dtype):
    """Strided float32 passes on the TMA-staged kernel (line counts that are
    multiples of 32): 2D columns with 512-sample windows and halos, whole
    lines up to 512, a 3D view (rank-3 tensor maps), in place; bit for bit
    against the oracle and against the kernels the option switches to."""
    rng = np.random.default_rng(26 + op)
    cases = [((4096, 64), [0], [6]), ((1024, 96), [0], [3]), ((2048, 32), [0], [1]),
             ((512, 64), [0], [4]), ((256, 32), [0], [5]), ((64, 32, 128), [0, 1], [3, 2]),
             ((96, 64), [1, 0], [2, 5])]
    for w in WAVELETS:
        for shape, axes, lv in cases:
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            if rc:
                continue
            g, _ = run(x, w, op, 0, axes, lv)
            assert np.array_equal(g, o), (w, shape, axes, lv)
            _lib.set_option("tma_strided", 0)
            try:
                g2, _ = run(x, w, op, 0, axes, lv)
            finally:
                _lib.set_option("tma_strided", 1)
            assert np.array_equal(g, g2)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_tma_long_strided_lines(op, dtype):
    """Long strided lines (windows with halos, the coarse levels on the
    approximation band in a second launch) with enough line groups for two
    lines per lane, a 3D view and more levels than the band launch holds in
    registers: bit for bit against the oracle."""
    rng = np.random.default_rng(40 + op)
    cases = [((4096, 2048), [0], [6]), ((2048, 32, 64), [0], [5]), ((4096, 64), [0], [9]),
             ((16384, 64), [0], [7]), ((8192, 32, 32), [0], [6])]
    for w in WAVELETS:
        for shape, axes, lv in cases:
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            if rc:
                continue
            g, _ = run(x, w, op, 0, axes, lv)
            assert np.array_equal(g, o), (w, shape, axes, lv)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_tma_stacked_short_lines(op, dtype):
    """Strided lines of 32 .. 256 samples in 3D views, several outer slices
    per staging window (outer extents that leave a last, partial group),
    and a 512-sample axis whose coarse band launch stacks: bit for bit
    against the oracle and against unstacked windows."""
    rng = np.random.default_rng(50 + op)
    cases = [((64, 40, 64), [0], [2]), ((32, 7, 96), [0], [1]), ((128, 3, 64), [0], [3]),
             ((256, 5, 128), [0], [4]), ((9, 64, 32), [1], [3]), ((512, 24, 64), [0], [4]),
             ((64, 64, 64), [0, 1, 2], [3, 3, 3])]
    for w in WAVELETS:
        for shape, axes, lv in cases:
            x = rng.standard_normal(shape).astype(dtype)
            rc, o = po.oracle_sep(x, w, op, 0, axes, lv)
            if rc:
                continue
            g, _ = run(x, w, op, 0, axes, lv)
            assert np.array_equal(g, o), (w, shape, axes, lv)
            _lib.set_option("tma_stacked", 0)
            try:
                g2, _ = run(x, w, op, 0, axes, lv)
            finally:
                _lib.set_option("tma_stacked", 1)
            assert np.array_equal(g2, o), (w, shape, axes, lv)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_long_rows_on_windows(op, dtype):
    """Contiguous rows longer than one warp holds, every level on windows
    with halos (first and last windows clipped by the row, a last window
    shorter than the others): bit for bit against the oracle and against
    the batch engine that serves them with the option off."""
    rng = np.random.default_rng(60 + op)
    cases = [((3, 65536), [2, 5]), ((2, 8192), [1, 4, 6]), ((4, 6080), [3]), ((1, 2112), [2, 5])]
    for w in WAVELETS:
        for shape, lvs in cases:
            for lv in lvs:
                x = rng.standard_normal(shape).astype(dtype)
                rc, o = po.oracle_sep(x, w, op, 0, [1], [lv])
                if rc:
                    continue
                g, _ = run(x, w, op, 0, [1], [lv])
                assert np.array_equal(g, o), (w, shape, lv)
                _lib.set_option("row_windows", 0)
                try:
                    g2, _ = run(x, w, op, 0, [1], [lv])
                finally:
                    _lib.set_option("row_windows", 1)
                assert np.array_equal(g2, o), (w, shape, lv)


def test_overlapped_launches_chain():
    """Back-to-back calls whose kernels are scheduled early and wait in
    hardware for the previous kernel (the overlap_launches option): a 2D
    forward then adjoint chain, later axes in place, equals the same chain
    with plain launches and the oracle."""
    rng = np.random.default_rng(28)
    x = rng.standard_normal((1024, 2048)).astype(np.float32)
    rc, want = po.oracle_sep(x, 100907, 0, 0, [0, 1], [6, 6])
    assert rc == 0
    rc, want2 = po.oracle_sep(want, 100907, 2, 0, [0, 1], [6, 6])
    assert rc == 0
    got = []
    for on in (1, 0):
        _lib.set_option("overlap_launches", on)
        try:
            t = torch.from_numpy(x).cuda()
            w = torch.empty_like(t)
            y = torch.empty_like(t)
            for op, a, b, ax in [(0, t, w, 0), (0, w, w, 1), (2, w, y, 0), (2, y, y, 1)]:
                pl._lwt(a, 100907, 0, op, (ax,), (6,), 1, out=b)
            got.append((w.cpu().numpy(), y.cpu().numpy()))
        finally:
            _lib.set_option("overlap_launches", 1)
    for w_, y_ in got:
        assert np.array_equal(w_, want) and np.array_equal(y_, want2)


def test_rows_two_warps_match_one_warp():
    """float32 rows of 2048 and 4096 split over two warps equal the
    one-warp-per-row kernel (option off) and the oracle."""
    rng = np.random.default_rng(27)
    for w in WAVELETS:
        for n in (2048, 4096):
            x = rng.standard_normal((5, n)).astype(np.float32)
            for tf in range(4):
                for lv in (1, 4, 6):
                    rc, o = po.oracle_sep(x, w, tf, 0, [1], [lv])
                    if rc:
                        continue
                    g, _ = run(x, w, tf, 0, [1], [lv])
                    _lib.set_option("wrow_split", 0)
                    try:
                        g2, _ = run(x, w, tf, 0, [1], [lv])
                    finally:
                        _lib.set_option("wrow_split", 1)
                    assert np.array_equal(g, o) and np.array_equal(g2, o), (w, n, tf, lv)
