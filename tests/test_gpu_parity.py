"""GPU parity: the CUDA library, called through its C ABI (lifted_b200's
pylifted entry points), against the reference's golden fixtures and the CPU
oracle.  The kernels restate the reference's Across-form arithmetic, so the
expected agreement is bit-exact in float32 and float64; the stated
tolerances (float64 1e-13 relative, float32 64 eps32 max|ref|) are only the
fallback bar for paths where the reference itself is not bitwise unique."""
import numpy as np
import pytest

import pyoracle as po
from helpers import REF_SHAPES, catalogue_cases, digest, fill_sin, load

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200 import pylifted as pl  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def cuda_ready():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    po.set_fold_order(True)
    _lib.set_option("force_global_scratch", 0)
    yield
    _lib.set_option("force_global_scratch", 0)


def gpu_sep(x, w, tf, bc, axes, levels):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    y = pl._lwt(t, w, bc, tf, axes, list(levels), 1)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def test_catalogue_golden_host_path():
    """Every wavelet x boundary x transform (f64 and f32), numpy in/out."""
    n = 0
    for w, bc, tf, lv, x, y in catalogue_cases():
        out = pl._lwt(x, w, bc, tf, [0], [lv], 1)
        assert np.array_equal(out, y), (w, bc, tf, x.dtype)
        n += 1
    assert n == 1360


def test_1d_sweep_vs_oracle_device_path():
    rng = np.random.default_rng(3)
    launches0 = _lib.launch_count()
    count = 0
    for dt in (np.float64, np.float32):
        for w in po.wavelet_values():
            width = po.wavelet_width(w)
            for n in (2, 3, 4, 7, 16, 33, 100, 255, 1024, 4097):
                ml = po.max_level(width, n) if width > 1 else int(np.log2(n))
                for lv in sorted({1, 2, max(ml, 1), ml + 2}):
                    if lv > 14:
                        continue
                    x = rng.standard_normal(n).astype(dt)
                    for bc in range(5):
                        for tf in range(4):
                            rc, o = po.oracle_sep(x, w, tf, bc, [0], [lv])
                            if rc:
                                with pytest.raises(_lib.LiftedValueError):
                                    gpu_sep(x, w, tf, bc, [0], [lv])
                                continue
                            g = gpu_sep(x, w, tf, bc, [0], [lv])
                            assert np.array_equal(g, o), (dt, w, n, lv, bc, tf)
                            count += 1
    assert count > 20000
    assert _lib.launch_count() - launches0 >= count


def test_nd_golden_digests():
    z = load("nd_shapes.npz")
    for (w, si, lv, bc, tf), (dsep, dnon) in zip(z["cases"], z["digests"]):
        shape, axes = REF_SHAPES[si]
        x = fill_sin(int(np.prod(shape)), -1524.421, 1643.32).reshape(shape)
        ys = pl._lwt(x, int(w), int(bc), int(tf), list(axes), [int(lv)] * len(axes), 1)
        assert digest(ys) == dsep, ("sep", w, shape, axes, lv, bc, tf)
        yn = pl._lwt(x, int(w), int(bc), int(tf), list(axes), int(lv), 1)
        assert digest(yn) == dnon, ("nonsep", w, shape, axes, lv, bc, tf)


@pytest.mark.parametrize("layout", ["C", "F", "neg", "inplace", "permuted"])
def test_nd_strides_vs_oracle(layout):
    rng = np.random.default_rng(5)
    for w in (2, 100907, 4, 10305):
        for shape, axes in REF_SHAPES:
            for bc in (0, 1, 2, 3, 4):
                for tf in range(4):
                    x = rng.standard_normal(shape)
                    lv = [2] * len(axes)
                    if layout == "F":
                        x = np.asfortranarray(x)
                    elif layout == "neg":
                        x = x[..., ::-1]
                    if layout == "inplace":
                        a = x.copy()
                        rc = po.oracle_sep(a, w, tf, bc, list(axes), lv, out=a)[0]
                        if rc:
                            continue
                        b = x.copy()
                        pl._lwt(b, w, bc, tf, list(axes), lv, 1, out=b)
                        assert np.array_equal(a, b)
                    elif layout == "permuted":
                        t = torch.from_numpy(x).cuda()
                        if t.ndim > 1:
                            t = t.transpose(0, -1)
                        xn = t.cpu().numpy()
                        rc, o = po.oracle_sep(xn, w, tf, bc, list(axes), lv)
                        if rc:
                            continue
                        out = torch.empty_like(t)
                        pl._lwt(t, w, bc, tf, list(axes), lv, 1, out=out)
                        assert np.array_equal(out.cpu().numpy(), o)
                    else:
                        rc, o = po.oracle_sep(x, w, tf, bc, list(axes), lv)
                        if rc:
                            continue
                        g = pl._lwt(x, w, bc, tf, list(axes), lv, 1)
                        assert np.array_equal(g, o), (w, shape, axes, bc, tf)
                    # non-separable on the same layout (host path)
                    if layout in ("C", "F", "neg"):
                        rc, o = po.oracle_nonsep(x, w, tf, bc, list(axes), 2)
                        if rc == 0:
                            g = pl._lwt(x, w, bc, tf, list(axes), 2, 1)
                            assert np.array_equal(g, o), ("nonsep", w, shape, axes, bc, tf)


def test_mock_step_programs():
    """The reference's 25 step-level programs (tests/test_single_levels.cpp)
    through the user-program entry point, one level on one line."""
    z = load("mock_steps.npz")
    for mi, prog in enumerate(po.MOCK_PROGRAMS):
        for ln in (153, 510):
            nd = ln // 2
            ns = ln - nd
            s0 = fill_sin(ns, -11.1, 13.4)
            d0 = fill_sin(nd, -10.2, 12.15)
            for bc in range(5):
                for tf in range(4):
                    if tf in (0, 3):   # forward-stepping: in = interleave, out = [s|d]
                        x = np.empty(ln)
                        x[0::2] = s0
                        x[1::2] = d0
                        y = pl.lwt_program(x, prog, tf, bc, axes=[0], level=[1])
                    else:              # reverse-stepping: in = [s|d], out interleaved
                        x = np.concatenate([s0, d0])
                        yi = pl.lwt_program(x, prog, tf, bc, axes=[0], level=[1])
                        y = np.concatenate([yi[0::2], yi[1::2]])
                    if ln == 153:
                        assert np.array_equal(y, z[f"m{mi}_{ln}_{bc}_{tf}"]), (mi, bc, tf)
                    else:
                        assert digest(y) == str(z[f"h{mi}_{ln}_{bc}_{tf}"]), (mi, bc, tf)


def test_global_scratch_path_matches_shared_path():
    rng = np.random.default_rng(9)
    _lib.set_option("force_global_scratch", 1)
    try:
        for w in (2, 100907, 203):
            for bc in range(5):
                for tf in range(4):
                    x = rng.standard_normal((5, 1000))
                    rc, o = po.oracle_sep(x, w, tf, bc, [1, 0], [4, 1])
                    if rc:
                        with pytest.raises(_lib.LiftedValueError):
                            gpu_sep(x, w, tf, bc, [1, 0], [4, 1])
                        continue
                    g = gpu_sep(x, w, tf, bc, [1, 0], [4, 1])
                    assert np.array_equal(g, o), (w, bc, tf)
    finally:
        _lib.set_option("force_global_scratch", 0)


def test_long_lines_global_path():
    """Lines too long for shared memory (f64 65536, f32 200000)."""
    rng = np.random.default_rng(10)
    for dt, n, w, lv in ((np.float64, 65536, 2, 5), (np.float32, 200003, 100907, 7)):
        for bc in (0, 2, 4):
            for tf in (0, 2):
                x = rng.standard_normal((2, n)).astype(dt)
                rc, o = po.oracle_sep(x, w, tf, bc, [1], [lv])
                g = gpu_sep(x, w, tf, bc, [1], [lv])
                assert rc == 0 and np.array_equal(g, o), (dt, n, bc, tf)


def test_host_and_device_paths_agree():
    rng = np.random.default_rng(13)
    x = rng.standard_normal((64, 96)).astype(np.float32)
    h = pl.lwt_forward(x, "cdf9.7", "Symmetric", axes=(0, 1), level=(3, 4))
    d = pl.lwt_forward(torch.from_numpy(x).cuda(), "cdf9.7", "Symmetric",
                       axes=(0, 1), level=(3, 4)).cpu().numpy()
    assert np.array_equal(h, d)


@pytest.mark.parametrize("tf", [0, 1, 2, 3])
def test_long_contiguous_lines_on_batch_engine(tf):
    """Contiguous lines too long for one CTA (Zero boundary) run on the batch
    engine, many CTAs per line; bit for bit against the oracle and against
    the single-CTA general kernel (option off); a second call reuses the
    cached plan."""
    rng = np.random.default_rng(40 + tf)
    for dt, shape, w, lv in ((np.float64, (4, 65536), 2, 5), (np.float32, (3, 100000), 10, 6),
                             (np.float64, (2, 3, 40000), 203, 4)):
        x = rng.standard_normal(shape).astype(dt)
        ax = len(shape) - 1
        rc, o = po.oracle_sep(x, w, tf, 0, [ax], [lv])
        assert rc == 0
        t = torch.from_numpy(x).cuda()
        for _ in range(2):
            n0 = _lib.launch_count()
            g = pl._lwt(t, w, 0, tf, (ax,), (lv,), 1).cpu().numpy()
            assert _lib.launch_count() - n0 == 1
            assert np.array_equal(g, o), (dt, shape, w)
        _lib.set_option("long_lines_batched", 0)
        try:
            g2 = pl._lwt(t, w, 0, tf, (ax,), (lv,), 1).cpu().numpy()
        finally:
            _lib.set_option("long_lines_batched", 1)
        assert np.array_equal(g2, o)
