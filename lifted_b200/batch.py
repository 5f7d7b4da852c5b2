"""Batched uneven-length 1D transforms: many signals, each with its own
length, wavelet and level count, in one persistent kernel launch.

The reference transforms one array per call (``pylifted.lwt_forward`` and
friends, src/pylifted/_wavelets.pyx:185-276); a batch there is a Python loop
of calls.  Here the signals are packed end to end in one flat CUDA tensor and
a plan (built once) cuts every signal into work items that one launch pulls
from a device queue.  Each signal's result equals the separable 1D transform
of that signal alone::

    plan = BatchPlan(lengths, wavelets, levels, op=Transform.Forward)
    y = plan.run(x)                 # x: flat float32 CUDA tensor
    y = plan.run(x, graph=True)     # replayed from a captured CUDA graph

The input and output must not overlap.  Runs are stream-ordered on torch's
current stream; ``plan.check()`` synchronises and raises if a bounded
device-side wait gave up.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _lib
from .pylifted import Transform, resolve_mode, resolve_wavelet

ITEM_FIELDS = ("kind", "prog", "sig", "lev0", "nlev", "src_sel", "dst_sel",
               "wait_ctr", "wait_target", "done_ctr", "n0", "in_off", "out_off",
               "src_off", "dst_off", "t0", "t1", "halo", "gbuf", "phase", "geo")
GEO_FIELDS = ("n", "sa", "oshape0", "oshape1", "oshape2", "ostride0", "ostride1", "ostride2")
KIND_NAMES = ("whole_fwd", "whole_rev", "tile_fwd", "tile_rev", "lines_fwd", "lines_rev")


def _torch():
    import torch

    return torch


def _dtype_bytes(dtype) -> int:
    name = str(dtype).replace("torch.", "")
    try:
        name = np.dtype(dtype).name
    except TypeError:
        pass
    if name in ("float32", "float", "f32"):
        return 4
    if name in ("float64", "double", "f64"):
        return 8
    raise TypeError(f"unsupported dtype {dtype}; float32 or float64")


def signal_table(lengths: Sequence[int], wavelets, levels=0, in_offsets=None,
                 out_offsets=None):
    """lifted_signal_t array.  Offsets default to the packed layout (signals
    end to end, the same offsets in and out)."""
    n = len(lengths)
    lengths = np.asarray(lengths, dtype=np.int64)
    if np.any(lengths < 0):
        raise ValueError("negative signal length")
    if isinstance(wavelets, (str, int)) or not hasattr(wavelets, "__len__"):
        wavelets = [wavelets] * n
    if np.ndim(levels) == 0:
        levels = [int(levels)] * n
    if len(wavelets) != n or len(levels) != n:
        raise ValueError("lengths, wavelets and levels differ in length")
    packed = np.concatenate([[0], np.cumsum(lengths)[:-1]]) if n else np.zeros(0, np.int64)
    ino = packed if in_offsets is None else np.asarray(in_offsets, dtype=np.int64)
    outo = ino if out_offsets is None else np.asarray(out_offsets, dtype=np.int64)
    tab = (_lib.Signal * max(n, 1))()
    for i in range(n):
        lv = int(levels[i])
        if lv < 0:
            raise ValueError(f"signal {i}: negative level")
        tab[i].wavelet = resolve_wavelet(wavelets[i])
        tab[i].levels = lv
        tab[i].length = int(lengths[i])
        tab[i].in_offset = int(ino[i])
        tab[i].out_offset = int(outo[i])
    return tab, n


class BatchPlan:
    """A planned batch (lifted_batch_plan_create_*)."""

    def __init__(self, lengths, wavelets, levels=0, op=Transform.Forward,
                 mode="Zero", dtype="float32", in_offsets=None, out_offsets=None,
                 tuning: dict | None = None):
        self._plan = ctypes.c_void_p()
        self.op = int(op)
        self.mode = resolve_mode(mode)
        self.dtype_bytes = _dtype_bytes(dtype)
        tab, n = signal_table(lengths, wavelets, levels, in_offsets, out_offsets)
        self.nsignals = n
        lengths = np.asarray(lengths, dtype=np.int64)
        ino = np.array([tab[i].in_offset for i in range(n)], dtype=np.int64)
        outo = np.array([tab[i].out_offset for i in range(n)], dtype=np.int64)
        self.in_elems = int((ino + lengths).max()) if n else 0
        self.out_elems = int((outo + lengths).max()) if n else 0
        tu = None
        if tuning:
            tu = _lib.BatchTuning(**{k: int(v) for k, v in tuning.items()})
        lib = _lib.load()
        fn = lib.lifted_batch_plan_create_f32 if self.dtype_bytes == 4 else \
            lib.lifted_batch_plan_create_f64
        _lib.check(fn(self.op, self.mode, n, ctypes.byref(tab),
                      ctypes.byref(tu) if tu is not None else None,
                      ctypes.byref(self._plan)))

    def _check_tensor(self, t, elems, what):
        torch = _torch()
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise TypeError(f"{what} must be a CUDA tensor")
        want = torch.float32 if self.dtype_bytes == 4 else torch.float64
        if t.dtype != want:
            raise TypeError(f"{what} has dtype {t.dtype}; the plan is for {want}")
        if not t.is_contiguous() or t.numel() < elems:
            raise ValueError(f"{what} must be contiguous with at least {elems} elements")

    def run(self, x, out=None, graph: bool = False, check: bool = False):
        """Transforms the packed signals of ``x`` into ``out`` (allocated as
        zeros of the output extent if not given) on the current stream."""
        torch = _torch()
        self._check_tensor(x, self.in_elems, "x")
        if out is None:
            out = torch.zeros(max(self.out_elems, 1), dtype=x.dtype, device=x.device)
        self._check_tensor(out, self.out_elems, "out")
        lib = _lib.load()
        with torch.cuda.device(x.device):
            stream = torch.cuda.current_stream(x.device).cuda_stream
            fn = lib.lifted_batch_run_graph if graph else lib.lifted_batch_run
            _lib.check(fn(self._plan, x.data_ptr(), out.data_ptr(), stream))
            if check:
                _lib.check(lib.lifted_batch_check(self._plan, stream))
        return out

    def check(self):
        torch = _torch()
        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.load().lifted_batch_check(self._plan, stream))

    @property
    def info(self) -> dict:
        inf = _lib.BatchInfo()
        _lib.check(_lib.load().lifted_batch_plan_info(self._plan, ctypes.byref(inf)))
        return {name: int(getattr(inf, name)) for name, _ in inf._fields_}

    def items(self) -> np.ndarray:
        """Work items in queue order, one row of ITEM_FIELDS each."""
        n = self.info["nitems"]
        out = np.zeros((n, len(ITEM_FIELDS)), dtype=np.int64)
        lib = _lib.load()
        buf = (ctypes.c_int64 * len(ITEM_FIELDS))()
        for i in range(n):
            _lib.check(lib.lifted_batch_plan_item(self._plan, i, buf, len(ITEM_FIELDS)))
            out[i] = np.frombuffer(buf, dtype=np.int64)
        return out

    def geometries(self) -> np.ndarray:
        """Axis-pass geometries of a plan of nD images, one row of GEO_FIELDS
        each (indexed by the line items' ``geo``)."""
        out = []
        lib = _lib.load()
        buf = (ctypes.c_int64 * len(GEO_FIELDS))()
        i = 0
        while lib.lifted_batch_plan_geo(self._plan, i, buf, len(GEO_FIELDS)) == _lib.OK:
            out.append(np.frombuffer(buf, dtype=np.int64).copy())
            i += 1
        return np.array(out, dtype=np.int64).reshape(-1, len(GEO_FIELDS))

    def close(self):
        if self._plan:
            _lib.load().lifted_batch_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def lwt_batch(x, lengths, wavelets, levels=0, op=Transform.Forward, mode="Zero",
              out=None):
    """One-shot batch transform of the packed signals of ``x`` (synchronous)."""
    plan = BatchPlan(lengths, wavelets, levels, op, mode, dtype=x.dtype)
    try:
        return plan.run(x, out=out, check=True)
    finally:
        plan.close()


def image_table(shapes, wavelets, levels=0, in_offsets=None, out_offsets=None):
    """lifted_image_t array for images of the given shapes (C order, 1..4
    axes).  ``levels``: one int for every axis of every image, or one entry
    per image (an int or a per-axis sequence).  Offsets default to the
    packed layout (images back to back, the same offsets in and out)."""
    n = len(shapes)
    if isinstance(wavelets, (str, int)) or not hasattr(wavelets, "__len__"):
        wavelets = [wavelets] * n
    if isinstance(levels, (int, np.integer)):
        levels = [int(levels)] * n
    if len(wavelets) != n or len(levels) != n:
        raise ValueError("shapes, wavelets and levels differ in length")
    sizes = [int(np.prod(s)) for s in shapes]
    packed = np.concatenate([[0], np.cumsum(sizes)[:-1]]) if n else np.zeros(0, np.int64)
    ino = packed if in_offsets is None else np.asarray(in_offsets, dtype=np.int64)
    outo = ino if out_offsets is None else np.asarray(out_offsets, dtype=np.int64)
    tab = (_lib.Image * max(n, 1))()
    for i, shp in enumerate(shapes):
        shp = tuple(int(v) for v in shp)
        if not 1 <= len(shp) <= 4:
            raise ValueError(f"image {i}: {len(shp)} axes; 1 to 4 supported")
        lv = levels[i]
        lv = [int(lv)] * len(shp) if isinstance(lv, (int, np.integer)) else [int(v) for v in lv]
        if len(lv) != len(shp) or min(lv) < 0:
            raise ValueError(f"image {i}: levels {lv} for shape {shp}")
        tab[i].wavelet = resolve_wavelet(wavelets[i])
        tab[i].ndim = len(shp)
        for d, v in enumerate(shp):
            tab[i].shape[d] = v
            tab[i].levels[d] = lv[d]
        tab[i].in_offset = int(ino[i])
        tab[i].out_offset = int(outo[i])
    return tab, n


class ImagePlan(BatchPlan):
    """A planned batch of nD images (lifted_batch_plan_create_nd_*): every
    image, a dense C-order array of 1..4 axes, is transformed separably over
    all of its axes; one persistent launch per run, whatever the shapes."""

    def __init__(self, shapes, wavelets, levels=0, op=Transform.Forward, mode="Zero",
                 dtype="float32", in_offsets=None, out_offsets=None,
                 tuning: dict | None = None):
        self._plan = ctypes.c_void_p()
        self.op = int(op)
        self.mode = resolve_mode(mode)
        self.dtype_bytes = _dtype_bytes(dtype)
        tab, n = image_table(shapes, wavelets, levels, in_offsets, out_offsets)
        self.nsignals = n
        sizes = np.array([int(np.prod(s)) for s in shapes], dtype=np.int64)
        ino = np.array([tab[i].in_offset for i in range(n)], dtype=np.int64)
        outo = np.array([tab[i].out_offset for i in range(n)], dtype=np.int64)
        self.in_elems = int((ino + sizes).max()) if n else 0
        self.out_elems = int((outo + sizes).max()) if n else 0
        tu = None
        if tuning:
            tu = _lib.BatchTuning(**{k: int(v) for k, v in tuning.items()})
        lib = _lib.load()
        fn = lib.lifted_batch_plan_create_nd_f32 if self.dtype_bytes == 4 else \
            lib.lifted_batch_plan_create_nd_f64
        _lib.check(fn(self.op, self.mode, n, ctypes.byref(tab),
                      ctypes.byref(tu) if tu is not None else None,
                      ctypes.byref(self._plan)))


def lwt_images(images, wavelets, levels=0, op=Transform.Forward, mode="Zero"):
    """Transforms a list of CUDA tensors of differing shapes (each separable
    over all of its axes, as ``pylifted`` would with ``axes=None``) in one C
    ABI call on the current stream: the images are packed into one buffer
    and run as one persistent launch, or, for a batch of a few distinct
    shapes, identically shaped neighbours as one launch per axis (the
    "batch_nd_mode" option).  Returns the list of results (views of one
    packed output)."""
    torch = _torch()
    if not images:
        return []
    dt = images[0].dtype
    dev = images[0].device
    for t in images:
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != dt or t.device != dev:
            raise TypeError("images must be CUDA tensors of one dtype on one device")
    shapes = [tuple(t.shape) for t in images]
    flat = torch.cat([t.reshape(-1) for t in images])
    out = torch.empty_like(flat)
    tab, n = image_table(shapes, wavelets, levels)
    lib = _lib.load()
    fn = lib.lifted_lwt_batch_nd_f32 if _dtype_bytes(dt) == 4 else lib.lifted_lwt_batch_nd_f64
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(fn(int(op), resolve_mode(mode), n, ctypes.byref(tab), flat.data_ptr(),
                      out.data_ptr(), stream))
    res, off = [], 0
    for shp in shapes:
        sz = int(np.prod(shp))
        res.append(out[off:off + sz].view(shp))
        off += sz
    return res


def autotune(wavelets, length: int, op=Transform.Forward, mode="Zero",
             dtype="float32", total: int = 1 << 24):
    """Runs the native autotuner for each wavelet at this signal length."""
    torch = _torch()
    ws = [resolve_wavelet(w) for w in wavelets]
    arr = (ctypes.c_uint32 * len(ws))(*ws)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.load().lifted_batch_autotune(_dtype_bytes(dtype), int(op),
                                                 resolve_mode(mode), len(ws), arr,
                                                 int(length), int(total), stream))


def tune_save(path: str):
    _lib.check(_lib.load().lifted_batch_tune_save(str(path).encode()))


def tune_load(path: str) -> int:
    n = ctypes.c_size_t(0)
    _lib.check(_lib.load().lifted_batch_tune_load(str(path).encode(), ctypes.byref(n)))
    return int(n.value)


def tune_clear():
    _lib.load().lifted_batch_tune_clear()
