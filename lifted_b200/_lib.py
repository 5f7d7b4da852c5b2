"""ctypes binding of liblifted_b200.so (the C ABI of include/lifted_capi.h).

The library is the product: there is no fallback.  If the shared object is
missing or cannot be loaded, importing the compute entry points raises.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "liblifted_b200.so"

OK = 0
EINVAL = 1
EDEGENERATE = 2
ENOTIMPL = 3
ECUDA = 4
ENOMEM = 5
ETIMEOUT = 6
ETOOLARGE = 7


class LiftedError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class LiftedValueError(LiftedError, ValueError):
    """Invalid argument, or an input on which the reference itself hangs or
    indexes out of bounds."""


class Step(ctypes.Structure):
    """lifted_step_t."""

    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("target", ctypes.c_uint32),
        ("offset", ctypes.c_int32),
        ("ntaps", ctypes.c_uint32),
        ("unit_sub", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("coef", ctypes.c_double * 9),
    ]


class Signal(ctypes.Structure):
    """lifted_signal_t."""

    _fields_ = [
        ("wavelet", ctypes.c_uint32),
        ("levels", ctypes.c_uint32),
        ("length", ctypes.c_uint64),
        ("in_offset", ctypes.c_uint64),
        ("out_offset", ctypes.c_uint64),
    ]


class Image(ctypes.Structure):
    """lifted_image_t."""

    _fields_ = [
        ("wavelet", ctypes.c_uint32),
        ("ndim", ctypes.c_uint32),
        ("shape", ctypes.c_uint64 * 4),
        ("levels", ctypes.c_uint32 * 4),
        ("in_offset", ctypes.c_uint64),
        ("out_offset", ctypes.c_uint64),
    ]


class BatchTuning(ctypes.Structure):
    """lifted_batch_tuning_t."""

    _fields_ = [
        ("block", ctypes.c_uint32),
        ("whole_max", ctypes.c_uint32),
        ("tile", ctypes.c_uint32),
        ("tile_levels", ctypes.c_uint32),
        ("spin_limit", ctypes.c_int32),
    ]


class BatchInfo(ctypes.Structure):
    """lifted_batch_info_t."""

    _fields_ = [(n, ctypes.c_uint64) for n in (
        "nsignals", "nitems", "ntiles", "nwhole", "nwhole_global", "ncounters",
        "scratch_bytes", "shared_bytes")] + [("grid", ctypes.c_uint32),
                                              ("block", ctypes.c_uint32)]


_lock = threading.Lock()
_lib = None

_sz = ctypes.c_size_t
_p = ctypes.c_void_p
_u32 = ctypes.c_uint32

# name -> (restype, argtypes)
_SIGS = {}
for _suf in ("f32", "f64"):
    _SIGS[f"lifted_lwt_sep_{_suf}"] = (ctypes.c_int, [_u32, _u32, _u32, _sz, _p, _p, _p, _sz, _p, _p, _p, _p, _p])
    _SIGS[f"lifted_lwt_{_suf}"] = (ctypes.c_int, [_u32, _u32, _u32, _sz, _p, _p, _p, _sz, _p, _sz, _p, _p, _p])
    _SIGS[f"lifted_lwt_sep_program_{_suf}"] = (ctypes.c_int, [_p, _sz, _sz, _u32, _u32, _sz, _p, _p, _p, _sz, _p, _p, _p, _p, _p])
_SIGS["lifted_lwt_sep_noalloc_f32"] = (ctypes.c_int, [_u32, _u32, _u32, _sz, _p, _p, _p, _sz, _p, _p, _p, _p, _p])
_SIGS["lifted_batch_plan_create_f32"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p])
_SIGS["lifted_batch_plan_create_f64"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p])
_SIGS["lifted_batch_run"] = (ctypes.c_int, [_p, _p, _p, _p])
_SIGS["lifted_batch_run_graph"] = (ctypes.c_int, [_p, _p, _p, _p])
_SIGS["lifted_batch_check"] = (ctypes.c_int, [_p, _p])
_SIGS["lifted_batch_plan_info"] = (ctypes.c_int, [_p, _p])
_SIGS["lifted_batch_plan_item"] = (ctypes.c_int, [_p, _sz, _p, _sz])
_SIGS["lifted_batch_plan_geo"] = (ctypes.c_int, [_p, _sz, _p, _sz])
_SIGS["lifted_batch_plan_destroy"] = (None, [_p])
_SIGS["lifted_lwt_batch_f32"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p, _p])
_SIGS["lifted_lwt_batch_f64"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p, _p])
_SIGS["lifted_batch_autotune"] = (ctypes.c_int, [_u32, _u32, _u32, _sz, _p, _sz, _sz, _p])
_SIGS["lifted_batch_tune_save"] = (ctypes.c_int, [ctypes.c_char_p])
_SIGS["lifted_batch_tune_load"] = (ctypes.c_int, [ctypes.c_char_p, _p])
_SIGS["lifted_batch_tune_clear"] = (None, [])
_SIGS["lifted_max_level"] = (_sz, [_sz, _sz])
_SIGS["lifted_wavelet_width"] = (_sz, [_u32])
_SIGS["lifted_wavelet_count"] = (_sz, [])
_SIGS["lifted_wavelet_value"] = (_u32, [_sz])
_SIGS["lifted_status_string"] = (ctypes.c_char_p, [ctypes.c_int])
_SIGS["lifted_last_error"] = (ctypes.c_char_p, [])
_SIGS["lifted_launch_count"] = (ctypes.c_uint64, [])
_SIGS["lifted_kernel_launch_count"] = (ctypes.c_uint64, [ctypes.c_char_p])
_SIGS["lifted_set_option"] = (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64])
_SIGS["lifted_device_check"] = (ctypes.c_int, [_p])
_SIGS["lifted_batch_plan_create_nd_f32"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p])
_SIGS["lifted_batch_plan_create_nd_f64"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p])
_SIGS["lifted_lwt_batch_nd_f32"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p, _p])
_SIGS["lifted_lwt_batch_nd_f64"] = (ctypes.c_int, [_u32, _u32, _sz, _p, _p, _p, _p])
_SIGS["lifted_blur2d_f32"] = (ctypes.c_int, [_p, _p, _sz, _sz, _sz, _p, _sz, ctypes.c_int, _p])

# Exported names the header declares (checked by the CPU test suite).
EXPORTED = tuple(_SIGS)


def load(path: str | os.PathLike | None = None):
    """Loads (once) and returns the shared library."""
    global _lib
    with _lock:
        if _lib is None:
            p = Path(path) if path else LIB_PATH
            if not p.exists():
                raise ImportError(
                    f"{p} is missing: build it with `python -m lifted_b200.build`")
            lib = ctypes.CDLL(str(p))
            for name, (res, args) in _SIGS.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def check(status: int) -> None:
    """Raises the Python exception matching a C ABI status."""
    if status == OK:
        return
    lib = load()
    msg = (lib.lifted_status_string(status) or b"").decode() + ": " + \
        (lib.lifted_last_error() or b"").decode()
    if status in (EINVAL, EDEGENERATE, ETOOLARGE):
        raise LiftedValueError(status, msg)
    if status == ENOMEM:
        raise MemoryError(msg)
    raise LiftedError(status, msg)


def launch_count() -> int:
    return int(load().lifted_launch_count())


def kernel_launches(family: str) -> int:
    """Launches of one kernel family so far ("line", "col", "wrow2", ...)."""
    return int(load().lifted_kernel_launch_count(family.encode()))


def set_option(name: str, value: int) -> None:
    check(load().lifted_set_option(name.encode(), int(value)))


def max_level(width: int, n: int) -> int:
    return int(load().lifted_max_level(width, n))


def wavelet_width(value: int) -> int:
    return int(load().lifted_wavelet_width(value))


def wavelet_values():
    lib = load()
    return [int(lib.lifted_wavelet_value(i)) for i in range(lib.lifted_wavelet_count())]
