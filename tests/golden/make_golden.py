#!/usr/bin/env python3
"""Generates tests/golden/*.npz from the reference implementation itself.

The reference (jcapriot/lifted) publishes no stored golden arrays; its
tests pin results by properties.  These fixtures are outputs of the
reference's own sources, compiled unchanged by oracle/build_ref.sh against
the Highway stand-in, on the one-lane build (every line takes the
reference's Across code path there).  Inputs are deterministic:
``fill_sin`` sinusoids as in the reference's tests/test_helpers.h:22-28 and
seeded normal draws.

Run from the repository root after oracle/build_ref.sh:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import pyoracle as po  # noqa: E402

OUT = Path(__file__).resolve().parent


def fill_sin(n, x0, xf, dtype=np.float64):
    """tests/test_helpers.h:22-28: sin(x0 + dx*i), dx = (xf-x0)/(n-1)."""
    dx = (xf - x0) / (n - 1)
    return np.sin(x0 + dx * np.arange(n)).astype(dtype)


def digest(a: np.ndarray) -> str:
    """SHA-256 of the exact bytes of a (C order): a bit-exact pin that stays
    small for the larger fixtures."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    if po.R("scalar") is None:
        raise SystemExit("reference build missing: run oracle/build_ref.sh")
    rng = np.random.default_rng(20261203)
    wavelets = po.wavelet_values()

    # 1. Every catalogue wavelet x boundary x transform, 1D, f64 and f32.
    rec = {"wavelet": [], "bc": [], "tf": [], "n": [], "level": [], "dtype": []}
    xs, ys = [], []
    for dt in (np.float64, np.float32):
        for w in wavelets:
            for bc in range(5):
                for tf in range(4):
                    n = 37 if dt == np.float64 else 50
                    lv = 2
                    x = rng.standard_normal(n).astype(dt)
                    rc, y = po.ref_sep(x, w, tf, bc, [0], [lv])
                    assert rc == 0
                    rec["wavelet"].append(w); rec["bc"].append(bc)
                    rec["tf"].append(tf); rec["n"].append(n)
                    rec["level"].append(lv); rec["dtype"].append(dt().itemsize)
                    xs.append(x.astype(np.float64)); ys.append(y.astype(np.float64))
    np.savez_compressed(OUT / "catalogue_1d.npz",
                        **{k: np.array(v) for k, v in rec.items()},
                        x=np.concatenate(xs), y=np.concatenate(ys))

    # 2. nD separable and non-separable: the shape/axes list of the
    #    reference's driver tests (tests/test_dwt.cpp:62-85), levels 1 and 3.
    shapes = [((31,), (0,)), ((32,), (0,)), ((32, 1), (0,)), ((1, 32), (1,)),
              ((34, 31), (1,)), ((23, 41), (0,)), ((34, 31), (1, 0)),
              ((23, 41), (0, 1)), ((25, 24, 31), (2,)), ((24, 23, 41), (1,)),
              ((24, 23, 41), (0,)), ((25, 24, 31), (2, 1)),
              ((24, 23, 41), (1, 0)), ((24, 23, 41), (0, 2)),
              ((23, 24, 31), (2, 1, 0))]
    cases = []
    digests = []
    samples = []
    for wname, w in (("db2", 2), ("cdf97", 100907)):
        for si, (shape, axes) in enumerate(shapes):
            for lv in (1, 3):
                for bc in (0, 2, 3):
                    for tf in range(4):
                        x = fill_sin(int(np.prod(shape)), -1524.421, 1643.32).reshape(shape)
                        rc, ys_ = po.ref_sep(x, w, tf, bc, list(axes), [lv] * len(axes))
                        assert rc == 0
                        rc2, yn = po.ref_nonsep(x, w, tf, bc, list(axes), lv)
                        assert rc2 == 0
                        cases.append((w, si, lv, bc, tf))
                        digests.append((digest(ys_), digest(yn)))
                        pick = np.linspace(0, ys_.size - 1, 8).astype(int)
                        samples.append(np.concatenate([ys_.ravel()[pick],
                                                       yn.ravel()[pick]]))
    np.savez_compressed(OUT / "nd_shapes.npz", cases=np.array(cases),
                        shapes=np.array([str(s_) for s_ in shapes]),
                        digests=np.array(digests), samples=np.array(samples))

    # 3. The 25 step-level programs of the reference's suite
    #    (tests/test_single_levels.cpp:82-412): FixedTransform::apply on
    #    pre-split bands of lengths 153 and 510, inputs as in the suite.
    steps = {}
    for mi in range(len(po.MOCK_PROGRAMS)):
        for ln in (153, 510):
            for bc in range(5):
                for tf in range(4):
                    nd = ln // 2
                    ns = ln - nd
                    s = fill_sin(ns, -11.1, 13.4)
                    d = fill_sin(nd, -10.2, 12.15)
                    rc = po.ref_fixed(s, d, tf, bc, 1, mi, direction=1)
                    assert rc == 0
                    y = np.concatenate([s, d])
                    if ln == 153:
                        steps[f"m{mi}_{ln}_{bc}_{tf}"] = y
                    else:
                        steps[f"h{mi}_{ln}_{bc}_{tf}"] = np.array(digest(y))
    np.savez_compressed(OUT / "mock_steps.npz", **steps)

    # 4. Known answer: db3 forward of a unit impulse at index 25 of a
    #    length-50 signal, Reflect, one level (the analysis filter taps).
    x = np.zeros(50)
    x[25] = 1.0
    rc, y = po.ref_sep(x, 3, 0, 4, [0], [1])
    assert rc == 0
    np.savez_compressed(OUT / "impulse_db3.npz", x=x, y=y)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
