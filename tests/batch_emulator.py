"""CPU emulation of a batch plan's work items (test infrastructure).

Runs the items of a lifted_batch plan in queue order on numpy arrays, with
the same window, interior and band bookkeeping as the CUDA batch kernel
(lifted_b200/csrc/lw_batch_kernel.cuh).  Every lifting step is the oracle's
FixedTransform::apply (pyoracle.oracle_fixed) on the split bands: on a whole
band that is the reference's driver; on a tile window it is the kernel's
tile step, whose taps count only inside the window, i.e. a Zero-boundary step
on the window arrays as a band of their own.  Comparing the emulated outputs
with the oracle's transform of each signal alone checks the planner (halo
sizes, group boundaries, scratch offsets, queue order) without a GPU.
"""
from __future__ import annotations

import numpy as np

import pyoracle as po
from lifted_b200.batch import ITEM_FIELDS, KIND_NAMES


def band_len(n, l):
    for _ in range(l):
        n -= n // 2
    return n


def _fixed(s, d, op, bc, wavelet):
    rc = po.oracle_fixed(s, d, op, bc, wavelet)
    assert rc == 0, rc


def emulate(items, op, bc, prog_wavelets, x, out_elems, scratch_elems, done=None, geos=None):
    """Runs the items; returns (out, scratch).  ``done`` collects completed
    counter increments to check every wait is satisfied when reached.
    ``geos``: the axis-pass geometries of a plan of nD images (line items:
    each line of the item is the oracle's 1D transform of that line, read
    from ``x`` for an image's first axis and in place from ``out`` after)."""
    dt = x.dtype
    out = np.zeros(max(out_elems, 1), dt)
    scratch = np.zeros(max(scratch_elems, 1), dt)
    arrs = {0: x, 1: out, 2: scratch}
    counters = {}
    for row in items:
        f = dict(zip(ITEM_FIELDS, (int(v) for v in row)))
        kind = KIND_NAMES[f["kind"]]
        w = prog_wavelets[f["prog"]]
        if f["wait_ctr"] >= 0:
            assert counters.get(f["wait_ctr"], 0) == f["wait_target"], \
                ("item runs before its producers", f)
        lev0, nlev = f["lev0"], f["nlev"]
        m = band_len(f["n0"], lev0)
        if kind in ("lines_fwd", "lines_rev"):
            g = geos[f["geo"]]
            n, sa, osh, ost = int(g[0]), int(g[1]), g[2:5], g[5:8]
            src = x[f["in_off"]:] if f["src_sel"] == 0 else out[f["out_off"]:]
            dst = out[f["out_off"]:]
            idx = np.arange(n) * sa
            for L in range(f["t0"], f["t1"]):
                i0, r = L % osh[0], L // osh[0]
                base = int(i0 * ost[0] + (r % osh[1]) * ost[1] + (r // osh[1]) * ost[2])
                line = src[base + idx].copy()
                rc, y = po.oracle_sep(line, w, op, bc, [0], [nlev])
                assert rc == 0, rc
                dst[base + idx] = y
        elif kind == "whole_fwd":
            src = arrs[f["src_sel"]]
            band = src[f["src_off"]:f["src_off"] + m].copy()
            region = np.empty(m, dt)
            for _ in range(nlev):
                s, d = band[0::2].copy(), band[1::2].copy()
                _fixed(s, d, op, bc, w)
                region[len(s):len(band)] = d
                band = s
            region[:len(band)] = band
            out[f["out_off"]:f["out_off"] + m] = region
        elif kind == "whole_rev":
            c = x[f["in_off"]:f["in_off"] + m]
            ml = [m]
            for _ in range(nlev):
                ml.append(ml[-1] - ml[-1] // 2)
            band = c[:ml[nlev]].copy()
            for j in range(nlev - 1, -1, -1):
                s, d = band, c[ml[j + 1]:ml[j]].copy()
                _fixed(s, d, op, bc, w)
                band = np.empty(ml[j], dt)
                band[0::2], band[1::2] = s, d
            dst = arrs[f["dst_sel"]]
            dst[f["dst_off"]:f["dst_off"] + m] = band
        elif kind == "tile_fwd":
            src = arrs[f["src_sel"]]
            wl0 = max(0, f["t0"] - f["halo"])
            wl1 = min(m, f["t1"] + f["halo"])
            win = src[f["src_off"] + wl0:f["src_off"] + wl1]
            S, D = win[0::2].copy(), win[1::2].copy()
            il0, il1 = f["t0"], min(f["t1"], m)
            for j in range(nlev):
                nd = m // 2
                ns = m - nd
                gb = wl0 >> 1
                assert wl0 % 2 == 0
                _fixed(S, D, op, bc, w)
                d_lo, d_hi = il0 >> 1, il1 >> 1
                out[f["out_off"] + ns + d_lo:f["out_off"] + ns + d_hi] = D[d_lo - gb:d_hi - gb]
                il0, il1 = il0 >> 1, (il1 + 1) >> 1
                wl0, wl1 = gb, gb + len(S)
                m = ns
                if j + 1 < nlev:
                    S, D = S[0::2].copy(), S[1::2].copy()
            dst = arrs[f["dst_sel"]]
            dst[f["dst_off"] + il0:f["dst_off"] + il1] = S[il0 - wl0:il1 - wl0]
        else:  # tile_rev
            ml = [m]
            wl1 = [min(m, f["t1"] + f["halo"])]
            W0 = max(0, f["t0"] - f["halo"])
            for j in range(nlev):
                ml.append(ml[j] - ml[j] // 2)
                wl1.append((wl1[j] + 1) >> 1)
            j = nlev - 1
            gb = (W0 >> j) >> 1
            src = arrs[f["src_sel"]]
            S = src[f["src_off"] + gb:f["src_off"] + wl1[j + 1]].copy()
            for j in range(nlev - 1, -1, -1):
                ns = ml[j + 1]
                wl0 = W0 >> j
                assert wl0 % 2 == 0
                gb = wl0 >> 1
                ndw = (wl1[j] - wl0) >> 1
                D = x[f["in_off"] + ns + gb:f["in_off"] + ns + gb + ndw].copy()
                assert len(S) == (wl1[j] - wl0 + 1) >> 1
                _fixed(S, D, op, bc, w)
                X = np.empty(wl1[j] - wl0, dt)
                X[0::2], X[1::2] = S, D
                if j > 0:
                    S = X
                else:
                    hi = min(f["t1"], ml[0])
                    dst = arrs[f["dst_sel"]]
                    dst[f["dst_off"] + f["t0"]:f["dst_off"] + hi] = X[f["t0"] - wl0:hi - wl0]
        if f["done_ctr"] >= 0:
            counters[f["done_ctr"]] = counters.get(f["done_ctr"], 0) + 1
    return out, scratch


def prog_wavelets(wavelets):
    """Program-table order of the planner: first appearance in signal order."""
    seen = []
    for w in wavelets:
        if w not in seen:
            seen.append(w)
    return seen
