"""ctypes access to the two CPU checkers.  TEST INFRASTRUCTURE ONLY.

* ``O``: the plain-C restatement of the reference algorithm
  (oracle/lifted_oracle.c, built into oracle/_build/liblifted_oracle.so).
* ``R``: the reference's own sources compiled against the Highway stand-in
  (oracle/build_ref.sh -> oracle/_ref/liblifted_ref_<variant>.so), present
  only where the reference tree was available at build time.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this
module.  Arrays are numpy; strides are converted to element units the way
pylifted does (``bytes // itemsize``, src/pylifted/_wavelets.pyx:243-248).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
O_PATH = HERE / "_build" / "liblifted_oracle.so"
R_DIR = HERE / "_ref"

OK, EINVAL, EDEGENERATE = 0, 1, 2

_c_size = ctypes.c_size_t
_c_ptr = ctypes.c_void_p
_u32 = ctypes.c_uint32


class UserStep(ctypes.Structure):
    """Layout of lo_user_step / lifted_step_t."""

    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("target", ctypes.c_uint32),
        ("offset", ctypes.c_int32),
        ("ntaps", ctypes.c_uint32),
        ("unit_sub", ctypes.c_uint32),
        ("pad_", ctypes.c_uint32),
        ("coef", ctypes.c_double * 9),
    ]


GEN, UNIT, REPEAT, SCALE = 0, 1, 2, 3
EVENS, ODDS = 0, 1


def make_program(steps):
    """steps: list of dicts {kind, target, offset, ntaps, unit_sub, coef}."""
    arr = (UserStep * max(1, len(steps)))()
    for i, st in enumerate(steps):
        arr[i].kind = st["kind"]
        arr[i].target = st.get("target", 0)
        arr[i].offset = st.get("offset", 0)
        coef = list(st.get("coef", []))
        arr[i].ntaps = st.get("ntaps", len(coef) if coef else 1)
        arr[i].unit_sub = st.get("unit_sub", 0)
        for k, c in enumerate(coef):
            arr[i].coef[k] = float(c)
    return arr, len(steps)


# The 25 single-step programs of the reference's step-level suite
# (tests/test_helpers.h:102-356), in MockWavelet order.
def _g(t, off, *c):
    return {"kind": GEN, "target": t, "offset": off, "coef": c}


def _u(t, off, sub):
    return {"kind": UNIT, "target": t, "offset": off, "unit_sub": sub, "ntaps": 1}


def _r(t, n, off, v):
    return {"kind": REPEAT, "target": t, "offset": off, "ntaps": n, "coef": [v]}


def _sc(*c):
    return {"kind": SCALE, "coef": c, "ntaps": len(c)}


MOCK_PROGRAMS = [
    [_g(EVENS, 0, 1.2)],
    [_g(EVENS, -5, 1.2, 1.5, 1.6)],
    [_g(EVENS, 3, 1.2, 1.5, 1.6)],
    [_g(EVENS, -2, 1.2, 1.3, 1.5, -1.2, -3.2)],
    [_g(ODDS, 0, 0.5)],
    [_g(ODDS, -5, 1.2, 1.5, 1.6)],
    [_g(ODDS, 3, 1.2, 1.5, 1.6)],
    [_g(ODDS, -2, 0.5, 1.203, 4.2, 33.213)],
    [_u(EVENS, 0, 0)],
    [_u(EVENS, 3, 1)],
    [_u(EVENS, -3, 0)],
    [_u(ODDS, 0, 1)],
    [_u(ODDS, 3, 0)],
    [_u(ODDS, -3, 1)],
    [_r(EVENS, 1, 0, 0.5)],
    [_r(EVENS, 3, -4, 0.5)],
    [_r(EVENS, 3, 2, 0.5)],
    [_r(EVENS, 3, -1, 0.5)],
    [_r(ODDS, 1, 0, 0.5)],
    [_r(ODDS, 3, -4, 0.5)],
    [_r(ODDS, 3, 2, 0.5)],
    [_r(ODDS, 3, -1, 0.5)],
    [_sc(0.124)],
    [_sc(5.23, 0.124)],
    [_g(EVENS, -5, 1.2, 1.3, 1.5, -1.2, -3.2),
     _g(ODDS, -5, 0.5, 1.203, 4.2, 33.213), _sc(0.124)],
]


def build_oracle() -> None:
    subprocess.run(["bash", str(HERE / "build_oracle.sh")], check=True)


_O = None


def O():
    """The C restatement (built on first use where gcc is available)."""
    global _O
    if _O is None:
        if not O_PATH.exists():
            build_oracle()
        lib = ctypes.CDLL(str(O_PATH))
        common = [_u32, _c_ptr, _c_size, _c_size, _u32, _u32, _c_size, _c_ptr,
                  _c_ptr, _c_ptr, _c_size, _c_ptr]
        for name in ("lo_sep_f32", "lo_sep_f64"):
            getattr(lib, name).argtypes = common + [_c_ptr, _c_ptr, _c_ptr]
            getattr(lib, name).restype = ctypes.c_int
        for name in ("lo_nonsep_f32", "lo_nonsep_f64"):
            getattr(lib, name).argtypes = common + [_c_size, _c_ptr, _c_ptr]
            getattr(lib, name).restype = ctypes.c_int
        for name in ("lo_fixed_apply_f32", "lo_fixed_apply_f64"):
            getattr(lib, name).argtypes = [_u32, _c_ptr, _c_size, _u32, _u32,
                                           _c_ptr, _c_ptr, _c_size, _c_size]
            getattr(lib, name).restype = ctypes.c_int
        lib.lo_set_fold_order.argtypes = [ctypes.c_int]
        lib.lo_wavelet_count.restype = _c_size
        lib.lo_wavelet_value.argtypes = [_c_size]
        lib.lo_wavelet_value.restype = _u32
        lib.lo_wavelet_width.argtypes = [_u32]
        lib.lo_wavelet_width.restype = _c_size
        lib.lo_max_level.argtypes = [_c_size, _c_size]
        lib.lo_max_level.restype = _c_size
        _O = lib
    return _O


_R = {}


def ref_variants():
    return [v for v in ("scalar", "avx2", "avx512")
            if (R_DIR / f"liblifted_ref_{v}.so").exists()]


def _cpu_flags() -> set:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def best_ref_variant():
    """Widest reference build this host can execute, or None."""
    flags = _cpu_flags()
    have = ref_variants()
    if "avx512" in have and {"avx512f", "avx512vl", "avx512dq", "avx512bw"} <= flags:
        return "avx512"
    if "avx2" in have and {"avx2", "fma"} <= flags:
        return "avx2"
    if "scalar" in have and {"avx2", "fma"} <= flags:
        return "scalar"
    return None


def R(variant: str = "scalar"):
    """The reference compiled from its own sources (None when absent)."""
    if variant not in _R:
        path = R_DIR / f"liblifted_ref_{variant}.so"
        if not path.exists():
            return None
        lib = ctypes.CDLL(str(path))
        common = [_u32, _u32, _u32, _c_size, _c_ptr, _c_ptr, _c_ptr, _c_size, _c_ptr]
        for name in ("ref_lwt_sep_f32", "ref_lwt_sep_f64"):
            getattr(lib, name).argtypes = common + [_c_ptr, _c_ptr, _c_ptr, _c_size]
            getattr(lib, name).restype = ctypes.c_int
        for name in ("ref_lwt_f32", "ref_lwt_f64"):
            getattr(lib, name).argtypes = common + [_c_size, _c_ptr, _c_ptr, _c_size]
            getattr(lib, name).restype = ctypes.c_int
        for name in ("ref_fixed_apply_f32", "ref_fixed_apply_f64"):
            getattr(lib, name).argtypes = [_u32, _u32, _u32, _u32, _u32, _c_ptr,
                                           _c_ptr, _c_size, _c_size]
            getattr(lib, name).restype = ctypes.c_int
        lib.ref_lanes_f32.restype = _c_size
        lib.ref_lanes_f64.restype = _c_size
        lib.ref_wavelet_width.argtypes = [_u32]
        lib.ref_wavelet_width.restype = _c_size
        lib.ref_max_level.argtypes = [_c_size, _c_size]
        lib.ref_max_level.restype = _c_size
        _R[variant] = lib
    return _R[variant]


def set_fold_order(across: bool) -> None:
    """Select the adjoint back-region order restated by the C oracle
    (True: the reference's Across form, the default)."""
    O().lo_set_fold_order(1 if across else 0)


def wavelet_values():
    lib = O()
    return [lib.lo_wavelet_value(i) for i in range(lib.lo_wavelet_count())]


def wavelet_width(w: int) -> int:
    return O().lo_wavelet_width(w)


def max_level(width: int, n: int) -> int:
    return O().lo_max_level(width, n)


def _arr(vals, ctype):
    vals = list(vals)
    return (ctype * max(1, len(vals)))(*vals)


def _geometry(x, out, axes):
    item = x.itemsize
    ndim = x.ndim
    shape = _arr(x.shape, ctypes.c_size_t)
    sin = _arr([s // item for s in x.strides], ctypes.c_ssize_t)
    sout = _arr([s // item for s in out.strides], ctypes.c_ssize_t)
    ax = _arr(axes, ctypes.c_size_t)
    return ndim, shape, sin, sout, ax


def _suffix(x):
    if x.dtype == np.float32:
        return "f32"
    if x.dtype == np.float64:
        return "f64"
    raise TypeError(f"unsupported dtype {x.dtype}")


def oracle_sep(x, wavelet, tf, bc, axes, levels, out=None, program=None, width=0):
    """Separable transform by the C restatement.  Returns (rc, out)."""
    if out is None:
        out = np.zeros_like(x)
    ndim, shape, sin, sout, ax = _geometry(x, out, axes)
    lv = _arr(levels, ctypes.c_size_t)
    prog, nprog = (None, 0) if program is None else make_program(program)
    fn = getattr(O(), "lo_sep_" + _suffix(x))
    rc = fn(wavelet, prog, nprog, width, tf, bc, ndim, shape, sin, sout,
            len(axes), ax, lv, x.ctypes.data, out.ctypes.data)
    return rc, out


def oracle_nonsep(x, wavelet, tf, bc, axes, level, out=None, program=None, width=0):
    if out is None:
        out = np.zeros_like(x)
    ndim, shape, sin, sout, ax = _geometry(x, out, axes)
    prog, nprog = (None, 0) if program is None else make_program(program)
    fn = getattr(O(), "lo_nonsep_" + _suffix(x))
    rc = fn(wavelet, prog, nprog, width, tf, bc, ndim, shape, sin, sout,
            len(axes), ax, level, x.ctypes.data, out.ctypes.data)
    return rc, out


def oracle_fixed(s, d, tf, bc, wavelet=0, program=None):
    """FixedTransform::apply on contiguous bands, in place.  Returns rc."""
    prog, nprog = (None, 0) if program is None else make_program(program)
    fn = getattr(O(), "lo_fixed_apply_" + _suffix(s))
    return fn(wavelet, prog, nprog, tf, bc, s.ctypes.data, d.ctypes.data,
              s.size, d.size)


def ref_sep(x, wavelet, tf, bc, axes, levels, out=None, variant="scalar", nthreads=1):
    lib = R(variant)
    if lib is None:
        raise FileNotFoundError("reference build not present (oracle/build_ref.sh)")
    if out is None:
        out = np.zeros_like(x)
    ndim, shape, sin, sout, ax = _geometry(x, out, axes)
    lv = _arr(levels, ctypes.c_size_t)
    fn = getattr(lib, "ref_lwt_sep_" + _suffix(x))
    rc = fn(wavelet, tf, bc, ndim, shape, sin, sout, len(axes), ax, lv,
            x.ctypes.data, out.ctypes.data, nthreads)
    return rc, out


def ref_nonsep(x, wavelet, tf, bc, axes, level, out=None, variant="scalar", nthreads=1):
    lib = R(variant)
    if lib is None:
        raise FileNotFoundError("reference build not present (oracle/build_ref.sh)")
    if out is None:
        out = np.zeros_like(x)
    ndim, shape, sin, sout, ax = _geometry(x, out, axes)
    fn = getattr(lib, "ref_lwt_" + _suffix(x))
    rc = fn(wavelet, tf, bc, ndim, shape, sin, sout, len(axes), ax, level,
            x.ctypes.data, out.ctypes.data, nthreads)
    return rc, out


def ref_fixed(s, d, tf, bc, kind, index, direction=0, variant="scalar"):
    """FixedTransform::apply by the reference (kind 0 catalogue wavelet value,
    kind 1 mock index); direction 0 Along, 1 Across."""
    lib = R(variant)
    fn = getattr(lib, "ref_fixed_apply_" + _suffix(s))
    lanes = (lib.ref_lanes_f32() if s.dtype == np.float32 else lib.ref_lanes_f64())
    ns = s.size // (lanes if direction else 1)
    nd = d.size // (lanes if direction else 1)
    return fn(kind, index, tf, direction, bc, s.ctypes.data, d.ctypes.data, ns, nd)


def nproc() -> int:
    return len(os.sched_getaffinity(0))
