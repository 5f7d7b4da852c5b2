"""The pylifted entry points on the B200 library.

Same names, arguments and results as the reference's Python package
(src/pylifted/__init__.py:1-8, src/pylifted/_wavelets.pyx:24-276):

    lwt_forward(x, wavelet, mode=BoundaryCondition.Zero, axes=None,
                level=1, n_threads=1, out=None)
    lwt_inverse(...), lwt_forward_adjoint(...), lwt_inverse_adjoint(...)
    Wavelet, BoundaryCondition, Transform

``level`` as an int selects the non-separable (Mallat) transform; a
sequence of ints, one per axis, the separable one (0 = max level).
``x`` may be a numpy array (host memory, staged through the GPU and
returned when done) or a torch tensor (CUDA tensors run on the current
stream without synchronising; CPU tensors are staged like numpy).
``out`` defaults to a new array of x's dtype and shape, Fortran-ordered
when x is.  ``n_threads`` is accepted and ignored.

Deviations from the reference, all on inputs where the reference misbehaves:
a dtype other than float32/float64 raises TypeError (the reference returns
the uninitialised ``out``); errors raise Python exceptions (the reference's
extern declarations lack ``except +``, so a C++ exception terminates the
process); an empty ``level`` sequence raises ValueError (the reference reads
an uninitialised level).
"""
from __future__ import annotations

import ctypes
import enum
import operator
from typing import Any, Sequence

import numpy as np

from . import _lib


class Wavelet(enum.IntEnum):
    """lifted::Wavelet (src/lifted-common.hpp:33-69)."""

    Lazy = 0
    Daubechies1 = 1
    Daubechies2 = 2
    Daubechies3 = 3
    Daubechies4 = 4
    Daubechies5 = 5
    Daubechies6 = 6
    Daubechies7 = 7
    Daubechies8 = 8
    Daubechies9 = 9
    Daubechies10 = 10
    Symlet4 = 104
    Symlet5 = 105
    Symlet6 = 106
    Coiflet2 = 202
    Coiflet3 = 203
    Bior1_3 = 10103
    Bior1_5 = 10105
    Bior2_2 = 10202
    Bior2_4 = 10204
    Bior2_6 = 10206
    Bior2_8 = 10208
    Bior3_1 = 10301
    Bior3_3 = 10303
    Bior3_5 = 10305
    Bior3_7 = 10307
    Bior3_9 = 10309
    Bior4_2 = 10402
    Bior4_4 = 10404
    Bior4_6 = 10406
    Bior5_5 = 10505
    Bior6_8 = 10608
    CDF5_3 = 100503
    CDF9_7 = 100907


class BoundaryCondition(enum.IntEnum):
    """lifted::BoundaryCondition (src/lifted-common.hpp:74-81)."""

    Zero = 0
    Constant = 1
    Periodic = 2
    Symmetric = 3
    Reflect = 4


class Transform(enum.IntEnum):
    """lifted::Transform (src/lifted-common.hpp:89-98)."""

    Forward = 0
    Inverse = 1
    ForwardAdjoint = 2
    InverseAdjoint = 3


# Name map of src/pylifted/_wavelets.pyx:101-140.
_MAP_STR_TO_WVLT = {
    "lazy": Wavelet.Lazy,
    "haar": Wavelet.Daubechies1,
    "db1": Wavelet.Daubechies1,
    "db2": Wavelet.Daubechies2,
    "db3": Wavelet.Daubechies3,
    "db4": Wavelet.Daubechies4,
    "db5": Wavelet.Daubechies5,
    "db6": Wavelet.Daubechies6,
    "db7": Wavelet.Daubechies7,
    "db8": Wavelet.Daubechies8,
    "db9": Wavelet.Daubechies9,
    "db10": Wavelet.Daubechies10,
    "sym1": Wavelet.Daubechies1,
    "sym2": Wavelet.Daubechies2,
    "sym3": Wavelet.Daubechies3,
    "sym4": Wavelet.Symlet4,
    "sym5": Wavelet.Symlet5,
    "sym6": Wavelet.Symlet6,
    "coif2": Wavelet.Coiflet2,
    "coif3": Wavelet.Coiflet3,
    "bior1.3": Wavelet.Bior1_3,
    "bior1.5": Wavelet.Bior1_5,
    "bior2.2": Wavelet.Bior2_2,
    "bior2.4": Wavelet.Bior2_4,
    "bior2.6": Wavelet.Bior2_6,
    "bior2.8": Wavelet.Bior2_8,
    "bior3.1": Wavelet.Bior3_1,
    "bior3.3": Wavelet.Bior3_3,
    "bior3.5": Wavelet.Bior3_5,
    "bior3.7": Wavelet.Bior3_7,
    "bior3.9": Wavelet.Bior3_9,
    "bior4.2": Wavelet.Bior4_2,
    "bior4.4": Wavelet.Bior4_4,
    "bior4.6": Wavelet.Bior4_6,
    "bior5.5": Wavelet.Bior5_5,
    "bior6.8": Wavelet.Bior6_8,
    "cdf5.3": Wavelet.CDF5_3,
    "cdf9.7": Wavelet.CDF9_7,
}


def resolve_wavelet(wavelet) -> int:
    """Enum member, its integer value, or a name of _MAP_STR_TO_WVLT
    (src/pylifted/_wavelets.pyx:229-235)."""
    if isinstance(wavelet, (int, np.integer)) and not isinstance(wavelet, bool):
        try:
            return int(Wavelet(int(wavelet)))
        except ValueError:
            raise KeyError(f"{wavelet} is not a valid Wavelet.") from None
    try:
        return int(_MAP_STR_TO_WVLT[wavelet])
    except (KeyError, TypeError):
        raise KeyError(f"{wavelet} is not a valid Wavelet.") from None


def resolve_mode(mode) -> int:
    """Enum member / value, or a case-sensitive member name
    (src/pylifted/_wavelets.pyx:238-241)."""
    if isinstance(mode, (int, np.integer)) and not isinstance(mode, bool):
        return int(BoundaryCondition(int(mode)))
    return int(BoundaryCondition[mode])


def get_axes(axes, ndim: int):
    """src/pylifted/_wavelets.pyx:142-166: None = every axis; negative axes
    wrap; an axis >= ndim raises ValueError."""
    if axes is None:
        axes = tuple(range(ndim))
    else:
        try:
            axes = tuple(axes)
        except TypeError:
            axes = (axes,)
    out = []
    for a in axes:
        try:
            a = operator.index(a)
        except TypeError as err:
            raise TypeError("Axes must be integers") from err
        if a >= ndim:
            raise ValueError(f"Axis {a} is beyond the array's dimensions, {ndim}.")
        if ndim == 0:
            raise ValueError("cannot transform a 0-d array")
        out.append(a % ndim)
    return out


def get_level(level, naxes: int):
    """src/pylifted/_wavelets.pyx:168-183: an int selects the non-separable
    transform, a sequence (one entry per axis) the separable one.
    Returns (level, levels) with exactly one of them not None."""
    try:
        lv = operator.index(level)
    except TypeError:
        try:
            levels = [operator.index(v) for v in level]
        except TypeError:
            raise TypeError("Level must be a single number, or a list of numbers") from None
        if len(levels) == 0:
            raise ValueError("levels must not be empty")
        if len(levels) != naxes:
            raise TypeError("levels must be the same length as axes")
        if any(v < 0 for v in levels):
            raise OverflowError("levels must be non-negative")
        return None, levels
    if lv < 0:
        raise OverflowError("level must be non-negative")
    return lv, None


def _is_torch(x) -> bool:
    mod = type(x).__module__
    return mod.startswith("torch")


def _arr(vals, ctype):
    vals = list(vals)
    return (ctype * max(1, len(vals)))(*vals)


def _call(op: int, wave: int, mode: int, shape, sin, sout, axes, level, levels,
          in_ptr: int, out_ptr: int, dtype_suffix: str, stream: int,
          program=None, width: int = 0) -> None:
    lib = _lib.load()
    ndim = len(shape)
    c_shape = _arr(shape, ctypes.c_size_t)
    c_sin = _arr(sin, ctypes.c_ssize_t)
    c_sout = _arr(sout, ctypes.c_ssize_t)
    c_axes = _arr(axes, ctypes.c_size_t)
    if program is not None:
        steps, nsteps = program
        c_lv = _arr(levels, ctypes.c_size_t)
        fn = getattr(lib, "lifted_lwt_sep_program_" + dtype_suffix)
        rc = fn(ctypes.cast(steps, ctypes.c_void_p), nsteps, width, op, mode,
                ndim, c_shape, c_sin, c_sout, len(axes), c_axes, c_lv, in_ptr,
                out_ptr, stream)
    elif levels is not None:
        c_lv = _arr(levels, ctypes.c_size_t)
        fn = getattr(lib, "lifted_lwt_sep_" + dtype_suffix)
        rc = fn(wave, op, mode, ndim, c_shape, c_sin, c_sout, len(axes), c_axes,
                c_lv, in_ptr, out_ptr, stream)
    else:
        fn = getattr(lib, "lifted_lwt_" + dtype_suffix)
        rc = fn(wave, op, mode, ndim, c_shape, c_sin, c_sout, len(axes), c_axes,
                level, in_ptr, out_ptr, stream)
    _lib.check(rc)


def make_program(steps: Sequence[dict]):
    """Builds a lifted_step_t array from dicts {kind, target, offset, ntaps,
    unit_sub, coef}; kind 0 generic, 1 unit, 2 repeat, 3 scale."""
    arr = (_lib.Step * max(1, len(steps)))()
    for i, st in enumerate(steps):
        coef = list(st.get("coef", []))
        arr[i].kind = int(st["kind"])
        arr[i].target = int(st.get("target", 0))
        arr[i].offset = int(st.get("offset", 0))
        arr[i].ntaps = int(st.get("ntaps", len(coef) if coef else 1))
        arr[i].unit_sub = int(st.get("unit_sub", 0))
        for k, c in enumerate(coef):
            arr[i].coef[k] = float(c)
    return arr, len(steps)


def _lwt(x, wavelet, mode, op: int, axes, level, n_threads, out=None,
         program=None, width: int = 0):
    """src/pylifted/_wavelets.pyx:185-264 over the C ABI."""
    ndim = x.ndim
    axes_ = get_axes(axes, ndim)
    level_, levels_ = get_level(level, len(axes_))
    if program is not None and levels_ is None:
        raise TypeError("a step program needs per-axis levels")
    wave = 0 if program is not None else resolve_wavelet(wavelet)
    mode_ = resolve_mode(mode)
    if _is_torch(x):
        import torch

        if x.dtype not in (torch.float32, torch.float64):
            raise TypeError(f"unsupported dtype {x.dtype}; float32 or float64")
        if out is None:
            if ndim > 1 and x.is_contiguous() is False and \
                    x.permute(*reversed(range(ndim))).is_contiguous():
                out = torch.empty(tuple(reversed(x.shape)), dtype=x.dtype,
                                  device=x.device).permute(*reversed(range(ndim)))
            else:
                out = torch.empty(x.shape, dtype=x.dtype, device=x.device)
        if out.dtype != x.dtype:
            raise ValueError(f"`out.dtype`:{out.dtype} does not match `input.dtype`:{x.dtype}.")
        if tuple(out.shape) != tuple(x.shape):
            for i in range(ndim):
                if out.shape[i] != x.shape[i]:
                    raise ValueError(f"`out.shape` does not match input along axis {i}.")
        if out.device != x.device:
            raise ValueError("`out` must be on the input's device")
        suffix = "f32" if x.dtype == torch.float32 else "f64"
        stream = 0
        if x.is_cuda:
            with torch.cuda.device(x.device):
                stream = torch.cuda.current_stream(x.device).cuda_stream
                _call(op, wave, mode_, tuple(x.shape), x.stride(), out.stride(),
                      axes_, level_, levels_, x.data_ptr(), out.data_ptr(),
                      suffix, stream, program, width)
        else:
            _call(op, wave, mode_, tuple(x.shape), x.stride(), out.stride(),
                  axes_, level_, levels_, x.data_ptr(), out.data_ptr(), suffix,
                  stream, program, width)
        return out

    x = np.asarray(x) if not isinstance(x, np.ndarray) else x
    if x.dtype not in (np.float32, np.float64):
        raise TypeError(f"unsupported dtype {x.dtype}; float32 or float64")
    if out is None:
        order = "F" if (x.flags.f_contiguous and not x.flags.c_contiguous) else "C"
        out = np.empty(x.shape, dtype=x.dtype, order=order)
    if out.dtype != x.dtype:
        raise ValueError(f"`out.dtype`:{out.dtype} does not match `input.dtype`:{x.dtype}.")
    for i in range(ndim):
        if x.shape[i] != out.shape[i]:
            raise ValueError(f"`out.shape` does not match input along axis {i}.")
    item = x.itemsize
    sin = [s // item for s in x.strides]
    sout = [s // item for s in out.strides]
    suffix = "f32" if x.dtype == np.float32 else "f64"
    _call(op, wave, mode_, x.shape, sin, sout, axes_, level_, levels_,
          x.ctypes.data, out.ctypes.data, suffix, 0, program, width)
    return out


def lwt_forward(x, wavelet, mode=BoundaryCondition.Zero, axes=None, level=1,
                n_threads=1, out=None):
    return _lwt(x, wavelet, mode, Transform.Forward, axes, level, n_threads, out=out)


def lwt_inverse(x, wavelet, mode=BoundaryCondition.Zero, axes=None, level=1,
                n_threads=1, out=None):
    return _lwt(x, wavelet, mode, Transform.Inverse, axes, level, n_threads, out=out)


def lwt_forward_adjoint(x, wavelet, mode=BoundaryCondition.Zero, axes=None,
                        level=1, n_threads=1, out=None):
    return _lwt(x, wavelet, mode, Transform.ForwardAdjoint, axes, level,
                n_threads, out=out)


def lwt_inverse_adjoint(x, wavelet, mode=BoundaryCondition.Zero, axes=None,
                        level=1, n_threads=1, out=None):
    return _lwt(x, wavelet, mode, Transform.InverseAdjoint, axes, level,
                n_threads, out=out)


def lwt_program(x, steps: Sequence[dict], op, mode=BoundaryCondition.Zero,
                axes=None, level: Any = None, out=None, width: int = 0):
    """Separable transform with a user step program (lifted_lwt_sep_program_*);
    ``level`` must be a per-axis sequence."""
    prog = make_program(steps)
    ndim = x.ndim
    naxes = len(get_axes(axes, ndim))
    if level is None:
        level = [1] * naxes
    return _lwt(x, None, mode, int(op), axes, level, 1, out=out, program=prog,
                width=width)
