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
