"""Batched nD images of differing shapes, wavelets and levels (one C ABI
call, lifted_lwt_batch_nd_*): every image bit for bit against the oracle's
separable transform of that image alone, packed groups and single images,
float32 and float64, all four transforms; argument checks."""
import ctypes

import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200.batch import image_table, lwt_images  # noqa: E402


def oracle_image(x, w, op, levels):
    rc, o = po.oracle_sep(x, w, op, 0, list(range(x.ndim)), list(levels))
    assert rc == 0
    return o


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_mixed_images_match_oracle(op, dtype):
    rng = np.random.default_rng(70 + op)
    spec = [((64, 96), 100907, (3, 4)), ((64, 96), 100907, (3, 4)), ((64, 96), 100907, (3, 4)),
            ((128, 128), 4, (2, 2)), ((96, 64), 2, (4, 2)), ((32, 16, 64), 100907, (2, 1, 3)),
            ((1000,), 6, (5,)), ((64, 96), 100907, (3, 4)), ((40, 24), 2, (0, 0))]
    xs = [rng.standard_normal(s).astype(dtype) for s, _, _ in spec]
    ys = lwt_images([torch.from_numpy(x).cuda() for x in xs], [w for _, w, _ in spec],
                    [lv for _, _, lv in spec], op=op)
    torch.cuda.synchronize()
    for x, y, (s, w, lv) in zip(xs, ys, spec):
        levels = [lv_ if lv_ else po.max_level(po.wavelet_width(w), n) for lv_, n in zip(lv, s)]
        assert np.array_equal(y.cpu().numpy(), oracle_image(x, w, op, levels)), (s, w, lv)


def test_groups_use_few_launches_and_checks():
    rng = np.random.default_rng(80)
    shapes = [(256, 256)] * 6 + [(128, 512)] * 2
    xs = [torch.from_numpy(rng.standard_normal(s).astype(np.float32)).cuda() for s in shapes]
    n0 = _lib.launch_count()
    ys = lwt_images(xs, "cdf9.7", 4)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - n0
    assert launches <= 8, launches  # two groups, a few launches per axis each
    for x, y in zip(xs, ys):
        assert np.array_equal(y.cpu().numpy(), oracle_image(x.cpu().numpy(), 100907, 0, (4, 4)))
    # overlapping outputs and host pointers are refused
    lib = _lib.load()
    tab, n = image_table([(16, 16), (16, 16)], "db2", 1, out_offsets=[0, 100])
    flat = torch.zeros(512, device="cuda")
    out = torch.zeros(512, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.lifted_lwt_batch_nd_f32(0, 0, n, ctypes.byref(tab), flat.data_ptr(),
                                       out.data_ptr(), s) == _lib.EINVAL
    tab, n = image_table([(16, 16)], "db2", 1)
    host = np.zeros(256, dtype=np.float32)
    assert lib.lifted_lwt_batch_nd_f32(0, 0, n, ctypes.byref(tab), host.ctypes.data,
                                       out.data_ptr(), s) == _lib.EINVAL
