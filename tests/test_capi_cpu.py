"""Host-side checks of the C ABI library that need no GPU: it loads, exports
every function include/lifted_capi.h declares, rejects invalid arguments
and the reference's hang/crash inputs exactly where the oracle does, and the
drop-in C++ header compiles against it and throws like the reference."""
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pyoracle as po
from lifted_b200 import _lib
from lifted_b200 import pylifted as pl

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "lifted_capi.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"LIFTED_CAPI\s+[\w\s\*]+?\b(lifted_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.EXPORTED)


def test_catalogue_queries_match_oracle():
    assert _lib.wavelet_values() == po.wavelet_values()
    for w in po.wavelet_values():
        assert _lib.wavelet_width(w) == po.wavelet_width(w)
    for width in (2, 4, 5, 9, 18, 21):
        for n in (0, 1, 3, 7, 8, 9, 100, 4096, 65536, 1 << 20):
            assert _lib.max_level(width, n) == po.max_level(width, n)


def _status(x, w, tf, bc, axes, levels, separable=True):
    lib = _lib.load()
    shape = (np.ctypeslib.ctypes.c_size_t * x.ndim)(*x.shape)
    st = (np.ctypeslib.ctypes.c_ssize_t * x.ndim)(*[s // x.itemsize for s in x.strides])
    ax = (np.ctypeslib.ctypes.c_size_t * max(1, len(axes)))(*axes)
    out = np.zeros_like(x)
    if separable:
        lv = (np.ctypeslib.ctypes.c_size_t * max(1, len(levels)))(*levels)
        return lib.lifted_lwt_sep_f64(w, tf, bc, x.ndim, shape, st, st, len(axes),
                                      ax, lv, x.ctypes.data, out.ctypes.data, None)
    return lib.lifted_lwt_f64(w, tf, bc, x.ndim, shape, st, st, len(axes), ax,
                              levels, x.ctypes.data, out.ctypes.data, None)


def test_invalid_arguments_rejected_without_gpu():
    x = np.zeros((4, 4))
    assert _status(x, 77, 0, 0, [0], [1]) == _lib.EINVAL      # unknown wavelet
    assert _status(x, 2, 4, 0, [0], [1]) == _lib.EINVAL       # unknown transform
    assert _status(x, 2, 0, 5, [0], [1]) == _lib.EINVAL       # unknown boundary
    assert _status(x, 2, 0, 0, [2], [1]) == _lib.EINVAL       # axis >= ndim
    assert _status(x, 0, 0, 0, [0], [0]) == _lib.EDEGENERATE  # Lazy, level 0
    assert _status(np.zeros((0, 3)), 2, 0, 0, [1], [1]) == _lib.OK  # empty
    assert _status(x, 2, 0, 0, [0], 0, separable=False) == _lib.EDEGENERATE


def test_degenerate_classification_matches_oracle():
    """The library refuses exactly the inputs on which the oracle detects a
    hang, division by zero or out-of-bounds access of the reference."""
    progs = [(w, None) for w in (0, 1, 2, 3, 100907, 10301, 10204)]
    progs += [(None, p) for p in po.MOCK_PROGRAMS]
    for w, prog in progs:
        for n in range(1, 9):
            for lv in (1, 2, 3, 5):
                x = np.zeros(n)
                for bc in range(5):
                    for tf in range(4):
                        if prog is None:
                            rc_o, _ = po.oracle_sep(x, w, tf, bc, [0], [lv])
                            rc_l = _status(x, w, tf, bc, [0], [lv])
                        else:
                            rc_o, _ = po.oracle_sep(x, 0, tf, bc, [0], [lv], program=prog)
                            try:
                                pl.lwt_program(x, prog, tf, bc, axes=[0], level=[lv])
                                rc_l = _lib.OK
                            except _lib.LiftedError as e:
                                rc_l = e.status
                        if rc_o == 2:
                            assert rc_l == _lib.EDEGENERATE, (w, n, lv, bc, tf)
                        else:
                            assert rc_l in (_lib.OK, _lib.ECUDA), (w, n, lv, bc, tf, rc_l)


def test_pylifted_argument_handling():
    assert pl.get_axes(None, 3) == [0, 1, 2]
    assert pl.get_axes(-1, 3) == [2]
    assert pl.get_axes((2, -3), 3) == [2, 0]
    with pytest.raises(ValueError):
        pl.get_axes(3, 3)
    with pytest.raises(TypeError):
        pl.get_axes(["a"], 3)
    assert pl.get_level(2, 2) == (2, None)
    assert pl.get_level([1, 0], 2) == (None, [1, 0])
    with pytest.raises(TypeError):
        pl.get_level([1], 2)
    with pytest.raises(TypeError):
        pl.get_level("x", 1)
    assert pl.resolve_wavelet("cdf9.7") == 100907
    assert pl.resolve_wavelet(pl.Wavelet.Daubechies2) == 2
    assert pl.resolve_wavelet(104) == 104
    with pytest.raises(KeyError):
        pl.resolve_wavelet("db11")
    assert pl.resolve_mode("Periodic") == 2
    assert pl.resolve_mode(pl.BoundaryCondition.Reflect) == 4
    with pytest.raises(KeyError):
        pl.resolve_mode("periodic")  # enum names are case-sensitive
    with pytest.raises(TypeError):
        pl.lwt_forward(np.zeros(8, dtype=np.int32), "db2")
    with pytest.raises(ValueError):
        pl.lwt_forward(np.zeros(8), "db2", out=np.zeros(8, dtype=np.float32))
    assert len(pl._MAP_STR_TO_WVLT) == 38


def test_options_hook():
    _lib.set_option("force_global_scratch", 1)
    _lib.set_option("force_global_scratch", 0)
    _lib.set_option("max_global_ctas", 296)
    with pytest.raises(_lib.LiftedValueError):
        _lib.set_option("no_such_option", 1)


CPP_TEST = r"""
#include <cstdio>
#include <stdexcept>
#include <vector>
#include "lifted.hpp"
int main() {
  using namespace lifted;
  std::vector<double> x(16, 1.0), y(16);
  int ok = 0;
  try {  // axis beyond the rank
    lwt(Wavelet::Daubechies2, Transform::Forward, BoundaryCondition::Zero,
        {16}, {1}, {1}, {1}, size_v{1}, x.data(), y.data());
  } catch (const std::invalid_argument&) { ok |= 1; }
  try {  // level 0 with the Lazy wavelet: the reference never returns
    lwt(Wavelet::Lazy, Transform::Forward, BoundaryCondition::Zero,
        {16}, {1}, {1}, {0}, size_v{0}, x.data(), y.data());
  } catch (const std::invalid_argument&) { ok |= 2; }
  try {  // levels shorter than axes
    lwt(Wavelet::CDF9_7, Transform::Forward, BoundaryCondition::Zero,
        {4, 4}, {4, 1}, {4, 1}, {0, 1}, size_v{1}, x.data(), y.data());
  } catch (const std::invalid_argument&) { ok |= 4; }
  if (max_level(9, 4096) != 9 || max_level(4, 65536) != 14) return 3;
  std::printf("%d\n", ok);
  return ok == 7 ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_dropin_header_compiles_links_and_throws(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(CPP_TEST)
    exe = tmp_path / "t"
    lib = _lib.LIB_PATH
    subprocess.run(["g++", "-std=c++20", "-O1", f"-I{ROOT / 'include'}", str(src),
                    "-o", str(exe), str(lib), f"-Wl,-rpath,{lib.parent}"],
                   check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
