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


@pytest.fixture
def nd_mode():
    yield lambda m: _lib.set_option("batch_nd_mode", m)
    _lib.set_option("batch_nd_mode", 0)


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_mixed_images_match_oracle(op, dtype, mode, nd_mode):
    """mode 1: one persistent launch of line items; mode 2: one separable
    call per group of identically shaped packed images."""
    nd_mode(mode)
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


def distinct_shapes(rng, count):
    """2D and 3D shapes, all different."""
    seen, out = set(), []
    while len(out) < count:
        if rng.random() < 0.8:
            shp = (int(rng.integers(40, 400)), int(rng.integers(40, 400)))
        else:
            shp = tuple(int(v) for v in rng.integers(40, 64, 3))
        if shp not in seen:
            seen.add(shp)
            out.append(shp)
    return out


@pytest.mark.parametrize("bc", [0, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_distinct_shapes_one_launch(op, dtype, bc, nd_mode):
    """48 images of 48 distinct shapes with mixed wavelets and levels: one
    launch per transform (the persistent batch kernel), every image bit for
    bit against the oracle's separable transform of it alone."""
    nd_mode(0)
    rng = np.random.default_rng(500 + op + 10 * bc)
    shapes = distinct_shapes(rng, 48)
    ws = [int(v) for v in rng.choice([2, 4, 100907, 5, 203, 10309], 48)]
    lvs = []
    for shp, w in zip(shapes, ws):
        # every axis at least one level (an axis of 0 levels leaves `out` as
        # it was, and lwt_images does not clear it)
        mxs = [po.max_level(po.wavelet_width(w), n) for n in shp]
        assert min(mxs) >= 1, (shp, w)
        lvs.append([int(rng.integers(1, mx + 1)) for mx in mxs])
    xs = [rng.standard_normal(s).astype(dtype) for s in shapes]
    ts = [torch.from_numpy(x).cuda() for x in xs]
    n0, b0 = _lib.launch_count(), _lib.kernel_launches("batch")
    ys = lwt_images(ts, ws, lvs, op=op, mode=bc)
    torch.cuda.synchronize()
    assert _lib.launch_count() - n0 == 1
    assert _lib.kernel_launches("batch") - b0 == 1
    for x, y, w, lv in zip(xs, ys, ws, lvs):
        rc, o = po.oracle_sep(x, w, op, bc, list(range(x.ndim)), lv)
        assert rc == 0
        assert np.array_equal(y.cpu().numpy(), o), (x.shape, w, lv)
    assert _lib.load().lifted_device_check(torch.cuda.current_stream().cuda_stream) == 0


def test_image_plan_graph_replay_in_place_and_global_slots():
    """A reusable plan of nD images: replayed from a CUDA graph, run in place
    (in == out), and with a shared-memory budget small enough that long
    lines work in per-CTA global slots."""
    from lifted_b200.batch import ImagePlan

    rng = np.random.default_rng(600)
    shapes = distinct_shapes(rng, 12)
    xs = [rng.standard_normal(s).astype(np.float32) for s in shapes]
    flat = np.concatenate([x.reshape(-1) for x in xs])
    want = []
    for x in xs:
        rc, o = po.oracle_sep(x, 100907, 0, 0, list(range(x.ndim)), [2] * x.ndim)
        want.append(o.reshape(-1))
    want = np.concatenate(want)
    for tuning in (None, {"whole_max": 64}):
        plan = ImagePlan(shapes, "cdf9.7", 2, op=0, dtype="float32", tuning=tuning)
        xt = torch.from_numpy(flat).cuda()
        out = plan.run(xt, graph=True, check=True)
        out = plan.run(xt, out=out, graph=True, check=True)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy()[:len(want)], want), tuning
        inplace = torch.from_numpy(flat).cuda()
        plan.run(inplace, out=inplace, check=True)
        torch.cuda.synchronize()
        assert np.array_equal(inplace.cpu().numpy(), want), tuning
        plan.close()
