"""Batch planner on the CPU: the work items of lifted_batch plans, executed
in queue order by the CPU emulator (tests/batch_emulator.py), reproduce the
oracle's transform of every signal alone, bit for bit; the queue puts every
producer group before its consumers; invalid batches are refused like the
separable entry refuses the same signal.  No GPU needed: a plan touches the
device only on its first run."""
import numpy as np
import pytest

import pyoracle as po
from batch_emulator import emulate, prog_wavelets
from lifted_b200 import _lib
from lifted_b200.batch import ITEM_FIELDS, KIND_NAMES, BatchPlan

# Daubechies2/4/10, Coiflet3, Bior3_9, CDF5_3, CDF9_7, Lazy, Symlet6, Bior6_8
WAVELETS = [2, 4, 10, 203, 10309, 100503, 100907, 0, 106, 10608]


def make_batch(seed, n, maxlen, dtype, levels_mode="random"):
    rng = np.random.default_rng(seed)
    lengths = rng.integers(1, maxlen, n)
    ws = [WAVELETS[i] for i in rng.integers(0, len(WAVELETS), n)]
    lv = []
    for L, w in zip(lengths, ws):
        width = po.wavelet_width(w)
        mx = int(np.floor(np.log2(L))) if width == 1 else po.max_level(width, int(L))
        mx = max(mx, 1)
        lv.append(int(rng.integers(1, mx + 1)) if levels_mode == "random" else mx)
    x = rng.standard_normal(int(lengths.sum())).astype(dtype)
    return lengths, ws, lv, x


def oracle_batch(x, lengths, ws, lv, op, bc):
    out = np.zeros_like(x)
    off = 0
    for L, w, l in zip(lengths, ws, lv):
        sig = x[off:off + L].copy()
        rc, o = po.oracle_sep(sig, w, op, bc, [0], [l])
        if rc == 0:
            out[off:off + L] = o
        off += L
    return out


@pytest.mark.parametrize("op", [0, 1, 2, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_emulated_tiles_match_oracle(op, dtype):
    lengths, ws, lv, x = make_batch(100 + op, 40, 3000, dtype)
    # small whole items and tiles force multi-group tiling on modest lengths
    for tuning in ({"whole_max": 256, "tile": 128},
                   {"whole_max": 200, "tile": 512, "tile_levels": 3},
                   {"whole_max": 64, "tile": 64, "tile_levels": 1}):
        plan = BatchPlan(lengths, ws, lv, op=op, mode="Zero", dtype=dtype, tuning=tuning)
        items = plan.items()
        info = plan.info
        assert info["ntiles"] > 0
        got, _ = emulate(items, op, 0, prog_wavelets(ws), x, plan.out_elems,
                         info["scratch_bytes"] // x.itemsize)
        want = oracle_batch(x, lengths, ws, lv, op, 0)
        assert np.array_equal(got[:len(want)], want), tuning
        plan.close()


@pytest.mark.parametrize("bc", [1, 2, 3, 4])
def test_other_boundaries_run_whole_items(bc):
    lengths, ws, lv, x = make_batch(7 + bc, 25, 1500, np.float64)
    plan = BatchPlan(lengths, ws, lv, op=2, mode=bc, dtype="float64",
                     tuning={"whole_max": 256})
    items = plan.items()
    kinds = {KIND_NAMES[k] for k in items[:, 0]}
    assert kinds <= {"whole_fwd", "whole_rev"}
    # bands beyond whole_max get global buffers
    assert plan.info["nwhole_global"] == int(np.sum(np.asarray(lengths) > 256))
    got, _ = emulate(items, 2, bc, prog_wavelets(ws), x, plan.out_elems,
                     plan.info["scratch_bytes"] // 8)
    want = oracle_batch(x, lengths, ws, lv, 2, bc)
    assert np.array_equal(got[:len(want)], want)


def test_queue_order_and_counters():
    lengths, ws, lv, x = make_batch(5, 60, 20000, np.float32, levels_mode="max")
    for op in (0, 2):
        plan = BatchPlan(lengths, ws, lv, op=op, dtype="float32",
                         tuning={"whole_max": 512, "tile": 1024})
        items = plan.items()
        f = {k: i for i, k in enumerate(ITEM_FIELDS)}
        produced = {}
        for row in items:
            if row[f["done_ctr"]] >= 0:
                produced[row[f["done_ctr"]]] = produced.get(row[f["done_ctr"]], 0) + 1
        seen = {}
        for row in items:
            if row[f["wait_ctr"]] >= 0:
                c = row[f["wait_ctr"]]
                # every producer of c is earlier in the queue
                assert seen.get(c, 0) == produced[c] == row[f["wait_target"]]
            if row[f["done_ctr"]] >= 0:
                seen[row[f["done_ctr"]]] = seen.get(row[f["done_ctr"]], 0) + 1
        # tiles are aligned to their level group
        for row in items:
            if KIND_NAMES[row[f["kind"]]].startswith("tile"):
                a = 1 << int(row[f["nlev"]])
                assert row[f["t0"]] % a == 0 and row[f["halo"]] % a == 0
        # phases never decrease along the queue
        assert np.all(np.diff(items[:, f["phase"]]) >= 0)
        plan.close()


def test_invalid_batches_refused():
    with pytest.raises(KeyError):
        BatchPlan([100], [12345], [1])          # unknown wavelet (pylifted's error)
    with pytest.raises(_lib.LiftedValueError):
        BatchPlan([100], [0], [0])              # Lazy with level 0 (Q14)
    with pytest.raises(_lib.LiftedValueError):
        BatchPlan([100], [2], [64])             # more than MAX_LEVELS
    with pytest.raises(_lib.LiftedValueError):
        BatchPlan([1], [2], [3], mode="Reflect")  # Reflect on a one-element band
    with pytest.raises(_lib.LiftedValueError):
        BatchPlan([100], [2], [1], tuning={"block": 100})
    # zero-length signals and zero resolved levels are no-ops
    p = BatchPlan([0, 3], [2, 4], [1, 0])
    assert p.info["nitems"] == 0
    p.close()


def test_tuning_table_round_trip_and_use(tmp_path):
    """A tuning entry for (wavelet, dtype, transform, log2 length) sets the
    tile width and levels per group of later plans; the table survives a
    save / load round trip as JSON."""
    from lifted_b200 import batch as bt

    bt.tune_clear()
    path = tmp_path / "tune.json"
    path.write_text('[\n  {"wavelet": 100907, "dtype_bytes": 4, "op": 0, "log2_length": 15, '
                    '"stride": 1, "tile": 1024, "tile_levels": 2, "us": 12.5}\n]\n')
    assert bt.tune_load(str(path)) == 1
    plan = BatchPlan([40000], [100907], [6], op=0, dtype="float32")
    items = plan.items()
    f = {k: i for i, k in enumerate(ITEM_FIELDS)}
    tiles = items[np.isin(items[:, f["kind"]], [2, 3])]
    assert len(tiles) > 0
    assert set(tiles[:, f["nlev"]].tolist()) <= {1, 2}
    assert (tiles[:, f["t1"]] - tiles[:, f["t0"]]).max() == 1024
    plan.close()
    out = tmp_path / "saved.json"
    bt.tune_save(str(out))
    bt.tune_clear()
    assert bt.tune_load(str(out)) == 1
    bt.tune_clear()


def random_images(seed, count, dtype):
    """Images of 1..4 axes and differing shapes, wavelets and per-axis
    levels (0 = max_level), packed back to back."""
    rng = np.random.default_rng(seed)
    shapes, ws, lvs = [], [], []
    for _ in range(count):
        nd = int(rng.integers(1, 5))
        shp = tuple(int(v) for v in rng.integers(3, {1: 300, 2: 70, 3: 20, 4: 9}[nd], nd))
        w = [v for v in WAVELETS if v != 0][int(rng.integers(0, len(WAVELETS) - 1))]
        # (not Lazy: its level 0 never resolves)
        width = po.wavelet_width(w)
        lv = []
        for n in shp:
            mx = po.max_level(width, n)
            lv.append(int(rng.integers(0, max(mx, 1) + 1)))
        shapes.append(shp)
        ws.append(w)
        lvs.append(lv)
    x = rng.standard_normal(int(sum(np.prod(s) for s in shapes))).astype(dtype)
    return shapes, ws, lvs, x


def oracle_images(x, shapes, ws, lvs, op, bc):
    out = np.zeros_like(x)
    off = 0
    for shp, w, lv in zip(shapes, ws, lvs):
        sz = int(np.prod(shp))
        img = x[off:off + sz].reshape(shp).copy()
        rc, o = po.oracle_sep(img, w, op, bc, list(range(len(shp))), lv)
        assert rc == 0, (shp, w, lv)
        out[off:off + sz] = o.reshape(-1)
        off += sz
    return out


@pytest.mark.parametrize("op", [0, 1, 2, 3])
@pytest.mark.parametrize("bc", [0, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_emulated_image_plan_matches_oracle(op, bc, dtype):
    """A plan of nD images of all-distinct shapes: its line items, run in
    queue order by the emulator (every wait satisfied by earlier items),
    give each image's separable transform over all of its axes; small
    shared-memory budgets force single lines and global slots."""
    from lifted_b200.batch import ImagePlan

    shapes, ws, lvs, x = random_images(300 + op + 10 * bc, 24, dtype)
    want = oracle_images(x, shapes, ws, lvs, op, bc)
    for tuning in (None, {"whole_max": 64}, {"whole_max": 16, "block": 64}):
        plan = ImagePlan(shapes, ws, lvs, op=op, mode=bc, dtype=dtype, tuning=tuning)
        items = plan.items()
        f = {k: i for i, k in enumerate(ITEM_FIELDS)}
        assert set(items[:, f["kind"]]) <= {4, 5}
        got, _ = emulate(items, op, bc, prog_wavelets(ws), x, plan.out_elems, 0,
                         geos=plan.geometries())
        assert np.array_equal(got[:len(want)], want), tuning
        if tuning and tuning["whole_max"] == 16:
            assert (items[:, f["gbuf"]] == -2).any()
        plan.close()


def test_image_plan_refuses_overlapping_outputs():
    from lifted_b200.batch import ImagePlan

    with pytest.raises(ValueError):
        ImagePlan([(8, 8), (8, 8)], "db2", 1, out_offsets=[0, 32])
