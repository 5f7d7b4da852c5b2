"""The persistent batch kernel against the oracle, bit for bit: uneven
signals with mixed wavelets and level counts, all four transforms, float32
and float64, small tiles (many groups, many waits) and the default planner;
replay from a captured CUDA graph; the one-shot C ABI entry; argument
checks."""
import ctypes

import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402
from lifted_b200.batch import BatchPlan, signal_table  # noqa: E402
from test_batch_plan import make_batch, oracle_batch  # noqa: E402


def run_plan(plan, x, graph=False):
    xt = torch.from_numpy(x).cuda()
    y = plan.run(xt, graph=graph, check=True)
    torch.cuda.synchronize()
    return y.cpu().numpy()[:len(x)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_small_tiles_match_oracle(op, dtype):
    lengths, ws, lv, x = make_batch(200 + op, 60, 6000, dtype)
    want = oracle_batch(x, lengths, ws, lv, op, 0)
    for tuning in ({"whole_max": 256, "tile": 128}, {"whole_max": 512, "tile": 1024},
                   {"whole_max": 64, "tile": 64, "tile_levels": 1, "block": 128}):
        plan = BatchPlan(lengths, ws, lv, op=op, dtype=dtype, tuning=tuning)
        assert plan.info["ntiles"] > 0
        got = run_plan(plan, x)
        assert np.array_equal(got, want), (tuning, np.argwhere(got != want)[:5])
        plan.close()


@pytest.mark.parametrize("op", [0, 2])
def test_uneven_lengths_all_wavelets_default_plan(op):
    rng = np.random.default_rng(31 + op)
    n = 120
    lengths = np.round(2.0 ** rng.uniform(8, 17, n)).astype(np.int64)
    allw = po.wavelet_values()
    ws = [allw[i] for i in rng.integers(0, len(allw), n)]
    lv = []
    for L, w in zip(lengths, ws):
        width = po.wavelet_width(w)
        mx = int(np.floor(np.log2(L))) if width == 1 else po.max_level(width, int(L))
        lv.append(int(rng.integers(1, max(mx, 1) + 1)))
    x = rng.standard_normal(int(lengths.sum())).astype(np.float32)
    want = oracle_batch(x, lengths, ws, lv, op, 0)
    plan = BatchPlan(lengths, ws, lv, op=op, dtype="float32")
    assert plan.info["ntiles"] > 0 and plan.info["nwhole"] > 0
    got = run_plan(plan, x)
    assert np.array_equal(got, want)
    # replayed from a CUDA graph, twice, and re-captured for new buffers
    g1 = run_plan(plan, x, graph=True)
    g2 = run_plan(plan, x, graph=True)
    assert np.array_equal(g1, want) and np.array_equal(g2, want)
    plan.close()


@pytest.mark.parametrize("bc", [1, 3])
def test_other_boundaries_whole_and_global_items(bc):
    lengths, ws, lv, x = make_batch(9 + bc, 30, 3000, np.float64)
    want = oracle_batch(x, lengths, ws, lv, 2, bc)
    plan = BatchPlan(lengths, ws, lv, op=2, mode=bc, dtype="float64",
                     tuning={"whole_max": 512})
    assert plan.info["nwhole_global"] > 0
    assert np.array_equal(run_plan(plan, x), want)
    plan.close()


def test_oneshot_c_abi_and_checks():
    lengths, ws, lv, x = make_batch(41, 20, 20000, np.float32)
    tab, n = signal_table(lengths, ws, lv)
    xt = torch.from_numpy(x).cuda()
    yt = torch.zeros_like(xt)
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.lifted_lwt_batch_f32(0, 0, n, ctypes.byref(tab), xt.data_ptr(),
                                  yt.data_ptr(), stream)
    assert rc == 0, _lib.load().lifted_last_error()
    assert np.array_equal(yt.cpu().numpy(), oracle_batch(x, lengths, ws, lv, 0, 0))
    # in place (overlapping input and output) and host pointers are refused
    rc = lib.lifted_lwt_batch_f32(0, 0, n, ctypes.byref(tab), xt.data_ptr(),
                                  xt.data_ptr(), stream)
    assert rc == _lib.EINVAL
    rc = lib.lifted_lwt_batch_f32(0, 0, n, ctypes.byref(tab), x.ctypes.data,
                                  yt.data_ptr(), stream)
    assert rc == _lib.EINVAL


def test_autotuner_records_a_choice_that_plans_use(tmp_path):
    """The autotuner times (tile width, levels per group) candidates on the
    GPU for a wavelet and length, records the fastest, and later plans with
    that key use it; results stay exact."""
    from lifted_b200 import batch as bt

    bt.tune_clear()
    bt.autotune(["cdf9.7", "db4"], 1 << 15, op=0, total=1 << 21)
    path = tmp_path / "tune.json"
    bt.tune_save(str(path))
    text = path.read_text()
    assert '"wavelet": 100907' in text and '"wavelet": 4' in text
    rng = np.random.default_rng(5)
    lengths = [1 << 15, 30000, 1 << 15]
    ws = [100907, 4, 100907]
    lv = [5, 4, 6]
    x = rng.standard_normal(sum(lengths)).astype(np.float32)
    plan = BatchPlan(lengths, ws, lv, op=0, dtype="float32")
    got = run_plan(plan, x)
    assert np.array_equal(got, oracle_batch(x, lengths, ws, lv, 0, 0))
    plan.close()
    bt.tune_clear()


def test_waits_that_run_out_report_timeout_and_leave_the_context_usable():
    """Failure detection without a GPU fault: with a spin limit of no polls,
    every item that waits for another item's band gives up at once; the
    kernel records the first such item, skips its work, lets its own
    dependents proceed and returns, and lifted_batch_check reports
    LIFTED_ETIMEOUT naming a waiting item.  The next run of a plan with the
    default limit is exact again."""
    import re

    from lifted_b200.batch import ITEM_FIELDS

    lengths, ws, lv, x = make_batch(240, 40, 6000, np.float32, levels_mode="max")
    tuning = {"whole_max": 256, "tile": 128, "tile_levels": 1, "spin_limit": -1}
    plan = BatchPlan(lengths, ws, lv, op=0, dtype="float32", tuning=tuning)
    items = plan.items()
    wait_col = ITEM_FIELDS.index("wait_ctr")
    waiting = set(np.flatnonzero(items[:, wait_col] >= 0).tolist())
    assert waiting, "the plan has no dependent items"
    xt = torch.from_numpy(x).cuda()
    plan.run(xt)
    lib = _lib.load()
    rc = lib.lifted_batch_check(plan._plan, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.ETIMEOUT
    m = re.search(r"batch item (\d+)", lib.lifted_last_error().decode())
    assert m and int(m.group(1)) in waiting
    plan.close()
    good = BatchPlan(lengths, ws, lv, op=0, dtype="float32",
                     tuning={"whole_max": 256, "tile": 128, "tile_levels": 1})
    got = run_plan(good, x)
    assert np.array_equal(got, oracle_batch(x, lengths, ws, lv, 0, 0))
    good.close()
