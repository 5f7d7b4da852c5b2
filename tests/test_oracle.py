"""The CPU oracle (oracle/lifted_oracle.c) pinned to the reference: golden
fixtures made by the reference's own sources, and, where the reference build
is present, a direct bit-exact sweep against it."""
import numpy as np
import pytest

import pyoracle as po
from helpers import REF_SHAPES, catalogue_cases, digest, fill_sin, load


@pytest.fixture(autouse=True)
def across_order():
    po.set_fold_order(True)
    yield
    po.set_fold_order(True)


def test_catalogue_golden_bit_exact():
    n = 0
    for w, bc, tf, lv, x, y in catalogue_cases():
        rc, o = po.oracle_sep(x, w, tf, bc, [0], [lv])
        assert rc == 0
        assert np.array_equal(o, y), (w, bc, tf, x.dtype)
        n += 1
    assert n == 2 * 34 * 5 * 4


def test_nd_golden_bit_exact():
    z = load("nd_shapes.npz")
    for (w, si, lv, bc, tf), (dsep, dnon), smp in zip(z["cases"], z["digests"], z["samples"]):
        shape, axes = REF_SHAPES[si]
        x = fill_sin(int(np.prod(shape)), -1524.421, 1643.32).reshape(shape)
        rc, ys = po.oracle_sep(x, int(w), int(tf), int(bc), list(axes), [int(lv)] * len(axes))
        assert rc == 0
        assert digest(ys) == dsep, ("sep", w, shape, axes, lv, bc, tf)
        rc, yn = po.oracle_nonsep(x, int(w), int(tf), int(bc), list(axes), int(lv))
        assert rc == 0
        pick = np.linspace(0, yn.size - 1, 8).astype(int)
        assert np.array_equal(yn.ravel()[pick], smp[8:])
        # the non-separable driver sends unit-stride output axes through the
        # reference's Along form (checked by digest as well)
        assert digest(yn) == dnon, ("nonsep", w, shape, axes, lv, bc, tf)


def test_mock_steps_golden():
    z = load("mock_steps.npz")
    for mi, prog in enumerate(po.MOCK_PROGRAMS):
        for ln in (153, 510):
            for bc in range(5):
                for tf in range(4):
                    nd = ln // 2
                    ns = ln - nd
                    s = fill_sin(ns, -11.1, 13.4)
                    d = fill_sin(nd, -10.2, 12.15)
                    assert po.oracle_fixed(s, d, tf, bc, program=prog) == 0
                    y = np.concatenate([s, d])
                    if ln == 153:
                        assert np.array_equal(y, z[f"m{mi}_{ln}_{bc}_{tf}"]), (mi, bc, tf)
                    else:
                        assert digest(y) == str(z[f"h{mi}_{ln}_{bc}_{tf}"]), (mi, bc, tf)


def test_impulse_db3_known_answer():
    z = load("impulse_db3.npz")
    rc, y = po.oracle_sep(z["x"], 3, 0, 4, [0], [1])
    assert rc == 0
    assert np.array_equal(y, z["y"])
    # the response of one level to an impulse is a pair of short filters
    assert np.count_nonzero(np.abs(y) > 1e-12) <= 12


def test_round_trip_and_adjoint_properties():
    rng = np.random.default_rng(7)
    for w in (2, 4, 100907, 10204, 104):
        for bc in range(5):
            x = rng.standard_normal(513)
            v = rng.standard_normal(513)
            _, wx = po.oracle_sep(x, w, 0, bc, [0], [4])
            _, back = po.oracle_sep(wx, w, 1, bc, [0], [4])
            np.testing.assert_allclose(back, x, rtol=0, atol=1e-9 * np.abs(x).max())
            _, wtv = po.oracle_sep(v, w, 2, bc, [0], [4])
            a, b = np.dot(v, wx), np.dot(wtv, x)
            assert abs(a - b) <= 1e-12 * max(abs(a), abs(b), 1.0)


def test_degenerate_inputs_flagged():
    x = np.zeros(1)
    assert po.oracle_sep(x, 2, 0, 2, [0], [1])[0] == 2      # Periodic, n=1
    assert po.oracle_sep(x, 2, 0, 3, [0], [1])[0] == 2      # Symmetric, n=1
    assert po.oracle_sep(np.zeros(2), 100907, 0, 4, [0], [1])[0] == 2  # Reflect, nx=1
    assert po.oracle_sep(np.zeros(8), 0, 0, 0, [0], [0])[0] == 2  # Lazy, level 0
    assert po.oracle_sep(x, 2, 0, 0, [0], [1])[0] == 0      # Zero is fine


@pytest.mark.skipif(po.R("scalar") is None, reason="reference build absent")
def test_oracle_matches_reference_sweep():
    rng = np.random.default_rng(11)
    wavelets = po.wavelet_values()
    checked = 0
    for dt in (np.float64, np.float32):
        for w in wavelets:
            for n in (2, 3, 5, 8, 17, 64, 99):
                for lv in (1, 3):
                    x = rng.standard_normal(n).astype(dt)
                    for bc in range(5):
                        for tf in range(4):
                            rc, o = po.oracle_sep(x, w, tf, bc, [0], [lv])
                            if rc:
                                continue  # the reference would hang or crash
                            rr, r = po.ref_sep(x, w, tf, bc, [0], [lv])
                            assert rr == 0
                            assert np.array_equal(o, r), (dt, w, n, lv, bc, tf)
                            checked += 1
    assert checked > 10000


@pytest.mark.skipif(po.R("scalar") is None, reason="reference build absent")
def test_oracle_matches_reference_strides():
    rng = np.random.default_rng(12)
    for w in (2, 100907):
        for shape, axes in REF_SHAPES[4:]:
            for layout in ("F", "neg", "inplace"):
                for tf in range(4):
                    x = rng.standard_normal(shape)
                    if layout == "F":
                        x = np.asfortranarray(x)
                    if layout == "neg":
                        x = x[..., ::-1]
                    if layout == "inplace":
                        a, b = x.copy(), x.copy()
                        assert po.oracle_sep(a, w, tf, 3, list(axes), [2] * len(axes), out=a)[0] == 0
                        assert po.ref_sep(b, w, tf, 3, list(axes), [2] * len(axes), out=b)[0] == 0
                        assert np.array_equal(a, b)
                    else:
                        rc, o = po.oracle_sep(x, w, tf, 3, list(axes), [2] * len(axes))
                        rr, r = po.ref_sep(x, w, tf, 3, list(axes), [2] * len(axes))
                        assert rc == rr == 0 and np.array_equal(o, r)
