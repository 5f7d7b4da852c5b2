"""Constant, Symmetric and Reflect boundaries on the fast kernels, bit for bit
against the oracle: the chunks holding a band's ends redo the edge elements
of every step in the reference's order (mapped taps for Forward and
Inverse, fold loops before and after the direct update for the adjoints,
src/lifted-steps-inl.hpp:409-615).  Strided passes on the TMA-staged kernel
(whole lines, windows with a chained band pass, 3D views), contiguous rows
on the warp-per-row kernel, the 2D benchmark image, and checks that no pass
fell back to the general kernel."""
import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200 import pylifted as pl  # noqa: E402

COMPILED = [2, 4, 100907]  # Daubechies2, Daubechies4, CDF9_7
BCS = [1, 3, 4]            # Constant, Symmetric, Reflect


def run(x, w, op, bc, axes, levels):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    l0 = _lib.kernel_launches("line")
    fams = ("col", "reg", "wrow", "wrow2")
    f0 = sum(_lib.kernel_launches(f) for f in fams)
    y = pl._lwt(t, w, bc, op, list(axes), list(levels), 1)
    torch.cuda.synchronize()
    fast = sum(_lib.kernel_launches(f) for f in fams) - f0
    return y.cpu().numpy(), _lib.kernel_launches("line") - l0, fast


def check(x, w, op, bc, axes, levels, want_fast):
    rc, o = po.oracle_sep(x, w, op, bc, list(axes), list(levels))
    if rc:
        return
    g, general, fast = run(x, w, op, bc, axes, levels)
    assert np.array_equal(g, o), (x.shape, w, op, bc, axes, levels,
                                  np.argwhere(g != o)[:4])
    if want_fast:
        assert general == 0 and fast > 0, (x.shape, w, op, bc, axes, levels, general, fast)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("bc", BCS)
def test_strided_passes(bc, dtype):
    rng = np.random.default_rng(700 + bc)
    cases = [((64, 64), 2), ((256, 96), 3), ((512, 64), 4), ((2048, 64), 5), ((4096, 64), 6),
             ((64, 8, 64), 3), ((1024, 4, 32), 4)]
    for w in COMPILED:
        width = po.wavelet_width(w)
        for shape, lv in cases:
            lv = max(1, min(lv, po.max_level(width, shape[0])))
            x = rng.standard_normal(shape).astype(dtype)
            for op in range(4):
                check(x, w, op, bc, [0], [lv], want_fast=(w == 100907 and shape[0] >= 256))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("bc", BCS)
def test_contiguous_rows_and_images(bc, dtype):
    rng = np.random.default_rng(710 + bc)
    for w in COMPILED:
        width = po.wavelet_width(w)
        for shape, axes, lv in [((6, 512), [1], [4]), ((3, 4096), [1], [6]),
                                ((256, 256), [0, 1], [3, 3]), ((32, 64, 128), [2, 0], [2, 3])]:
            lv = [max(1, min(l_, po.max_level(width, shape[a]))) for a, l_ in zip(axes, lv)]
            x = rng.standard_normal(shape).astype(dtype)
            for op in range(4):
                check(x, w, op, bc, axes, lv, want_fast=(w == 100907))


@pytest.mark.parametrize("bc", BCS)
def test_benchmark_image_cdf97_fast(bc):
    """4096^2 float32 CDF 9/7, levels (6, 6): every transform exact, every
    pass on the fast kernels."""
    rng = np.random.default_rng(720 + bc)
    x = rng.standard_normal((4096, 4096)).astype(np.float32)
    for op in range(4):
        check(x, 100907, op, bc, [0, 1], [6, 6], want_fast=True)


def test_periodic_stays_exact_on_the_general_kernel():
    rng = np.random.default_rng(730)
    x = rng.standard_normal((512, 256)).astype(np.float32)
    for op in range(4):
        rc, o = po.oracle_sep(x, 100907, op, 2, [0, 1], [3, 3])
        g, general, _ = run(x, 100907, op, 2, [0, 1], [3, 3])
        assert np.array_equal(g, o) and general > 0
