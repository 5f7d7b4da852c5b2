"""Shared test helpers: fixture loading and input generators."""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

# The shape/axes list of the reference's driver tests (tests/test_dwt.cpp:62-85).
REF_SHAPES = [((31,), (0,)), ((32,), (0,)), ((32, 1), (0,)), ((1, 32), (1,)),
              ((34, 31), (1,)), ((23, 41), (0,)), ((34, 31), (1, 0)),
              ((23, 41), (0, 1)), ((25, 24, 31), (2,)), ((24, 23, 41), (1,)),
              ((24, 23, 41), (0,)), ((25, 24, 31), (2, 1)),
              ((24, 23, 41), (1, 0)), ((24, 23, 41), (0, 2)),
              ((23, 24, 31), (2, 1, 0))]


def fill_sin(n, x0, xf, dtype=np.float64):
    """tests/test_helpers.h:22-28 of the reference."""
    dx = (xf - x0) / (n - 1)
    return np.sin(x0 + dx * np.arange(n)).astype(dtype)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load(name: str):
    return np.load(GOLDEN / name, allow_pickle=False)


def catalogue_cases():
    """Yields (wavelet, bc, tf, level, x, y_golden) from catalogue_1d.npz."""
    z = load("catalogue_1d.npz")
    off = 0
    for w, bc, tf, n, lv, item in zip(z["wavelet"], z["bc"], z["tf"], z["n"],
                                      z["level"], z["dtype"]):
        dt = np.float64 if item == 8 else np.float32
        x = z["x"][off:off + n].astype(dt)
        y = z["y"][off:off + n].astype(dt)
        off += n
        yield int(w), int(bc), int(tf), int(lv), x, y


def f32_bound(ref: np.ndarray) -> float:
    """The stated float32 tolerance: max|delta| <= 64 * eps32 * max|ref|."""
    return 64 * np.finfo(np.float32).eps * float(np.max(np.abs(ref)) or 1.0)
