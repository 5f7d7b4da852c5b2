"""Sharding across ranks, on the CPU with the gloo backend (world size 2):
each rank plans its shard of an uneven batch (no GPU needed to plan), runs
the plan's work items with the CPU emulator, and the gathered shards equal
the oracle's transform of the whole batch; the max-over-ranks timing helper
returns the same value on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lifted_b200.shard import rank_batch, shard_signals


def test_shard_boundaries_balance_samples():
    rng = np.random.default_rng(0)
    lengths = np.round(2.0 ** rng.uniform(8, 16, 500)).astype(np.int64)
    for world in (1, 2, 3, 8):
        b = shard_signals(lengths, world)
        assert b[0] == 0 and b[-1] == len(lengths) and all(np.diff(b) >= 0)
        per = [int(lengths[b[r]:b[r + 1]].sum()) for r in range(world)]
        assert sum(per) == int(lengths.sum())
        assert max(per) - min(per) <= 2 * int(lengths.max())
    assert shard_signals([], 2) == [0, 0, 0]
    with pytest.raises(ValueError):
        shard_signals([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    import pyoracle as po
    from batch_emulator import emulate, prog_wavelets
    from lifted_b200.batch import BatchPlan
    from lifted_b200.shard import max_over_ranks
    from test_batch_plan import make_batch

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lengths, ws, lv, x = make_batch(77, 30, 4000, np.float32)
        lo, hi, L, W, V, off = rank_batch(lengths, ws, lv, rank, world)
        xs = x[off:off + int(L.sum())]
        plan = BatchPlan(L, W, V, op=0, dtype="float32",
                         tuning={"whole_max": 256, "tile": 256})
        out, _ = emulate(plan.items(), 0, 0, prog_wavelets(W), xs, plan.out_elems,
                         plan.info["scratch_bytes"] // 4)
        plan.close()
        mine = torch.from_numpy(out[:len(xs)].copy())
        sizes = [None] * world
        dist.all_gather_object(sizes, int(len(xs)))
        mx = max(sizes)
        parts = [torch.zeros(mx, dtype=torch.float32) for _ in sizes]
        dist.all_gather(parts, torch.nn.functional.pad(mine, (0, mx - len(xs))))
        parts = [p[:s] for p, s in zip(parts, sizes)]
        t = max_over_ranks(float(rank + 1))
        if rank == 0:
            full = np.concatenate([p.numpy() for p in parts])
            want = np.zeros_like(x)
            o = 0
            for n_, w_, l_ in zip(lengths, ws, lv):
                rc, y = po.oracle_sep(x[o:o + n_].copy(), w_, 0, 0, [0], [l_])
                want[o:o + n_] = y
                o += n_
            q.put((bool(np.array_equal(full, want)), t))
        else:
            q.put((True, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_a_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=60) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for ok, _ in res)
    assert all(t == 2.0 for _, t in res)
