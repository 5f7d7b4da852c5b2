"""The entry point that allocates nothing (lifted_lwt_sep_noalloc_f32),
called through the C ABI and checked against the regular entry point
(lifted_lwt_sep_f32) on the same inputs, twice in a row.

It exists for callers that must not allocate device memory (an application
that owns the GPU's memory and forbids its plugins from calling cudaMalloc,
or a latency-critical loop).  Long lines use its fixed static scratch array
instead of a stream-ordered allocation; the second call checks that the
array's leftover contents from the first call do not leak into the result.
This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402


def _call(fn, x, w, tf, bc, axes, levels, out):
    lib = _lib.load()
    shape = (ctypes.c_size_t * x.ndim)(*x.shape)
    sin = (ctypes.c_ssize_t * x.ndim)(*x.stride())
    sout = (ctypes.c_ssize_t * x.ndim)(*out.stride())
    ax = (ctypes.c_size_t * len(axes))(*axes)
    lv = (ctypes.c_size_t * len(levels))(*levels)
    stream = torch.cuda.current_stream().cuda_stream
    return getattr(lib, fn)(w, tf, bc, x.ndim, shape, sin, sout, len(axes), ax,
                            lv, x.data_ptr(), out.data_ptr(), stream)


# (shape, axes, levels, wavelet, boundary): short lines (shared memory) and
# lines too long for shared memory (static scratch), several boundaries.
CASES = [
    ((64, 256), (1, 0), (4, 3), 100907, 0),
    ((4, 200003), (1,), (7,), 100907, 3),
    ((3, 65536), (1,), (5,), 2, 2),
    ((70000, 2), (0,), (6,), 4, 4),
]


@pytest.mark.parametrize("case", CASES)
def test_noalloc_matches_regular_entry_twice(case):
    shape, axes, levels, w, bc = case
    assert torch.cuda.is_available()
    torch.manual_seed(7)
    for tf in (0, 2):
        x = torch.randn(*shape, device="cuda", dtype=torch.float32)
        ref = torch.empty_like(x)
        assert _call("lifted_lwt_sep_f32", x, w, tf, bc, axes, levels, ref) == 0
        for _ in range(2):
            out = torch.full_like(x, float("nan"))
            rc = _call("lifted_lwt_sep_noalloc_f32", x, w, tf, bc, axes, levels, out)
            assert rc == 0, _lib.load().lifted_last_error()
            torch.cuda.synchronize()
            assert torch.equal(out, ref), (case, tf)


def test_noalloc_rejects_oversized_lines_and_host_pointers():
    n = (32 << 20) // 6 + 64          # longer than the static array can hold
    x = torch.zeros(1, n, device="cuda", dtype=torch.float32)
    out = torch.empty_like(x)
    assert _call("lifted_lwt_sep_noalloc_f32", x, 2, 0, 0, (1,), (1,), out) == _lib.ETOOLARGE
    assert "scratch" in _lib.load().lifted_last_error().decode()
    lib = _lib.load()
    h = np.zeros((4, 8), np.float32)
    ho = np.zeros_like(h)
    shape = (ctypes.c_size_t * 2)(4, 8)
    st = (ctypes.c_ssize_t * 2)(8, 1)
    ax = (ctypes.c_size_t * 1)(1)
    lv = (ctypes.c_size_t * 1)(1)
    rc = lib.lifted_lwt_sep_noalloc_f32(2, 0, 0, 2, shape, st, st, 1, ax, lv,
                                        h.ctypes.data, ho.ctypes.data, None)
    assert rc == _lib.EINVAL
