"""Multi-process sharding on CPU (gloo, world size 2): partitioning, the
gather back into input order, and max-over-ranks timing.  The per-rank
compute is the oracle, so no GPU is involved."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from periodfind_b200.distributed import partition_by_work


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    lengths = np.clip(rng.lognormal(np.log(300), 0.8, 1000).astype(int), 20, 2000)
    parts = partition_by_work(lengths, 4)
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(1000))
    loads = [lengths[p].sum() for p in parts]
    assert max(loads) - min(loads) <= lengths.max()


def test_partition_more_ranks_than_curves():
    parts = partition_by_work([5, 3], 4)
    assert sorted(np.concatenate(parts).tolist()) == [0, 1]
    assert sum(len(p) == 0 for p in parts) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from oracle import oracle as O
    from periodfind_b200.distributed import calc_sharded, max_over_ranks
    import lightcurves as lc

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(3)
        ts, ms = [], []
        for n in (50, 700, 33, 400, 1200, 8, 90):
            t = lc.uniform_times(rng, n, 300.0)
            ts.append(t)
            ms.append(lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(1, 5))), 0.05))
        periods = np.linspace(0.5, 6.0, 64, dtype=np.float32)
        pdts = np.zeros(1, np.float32)
        compute = lambda t, m: list(O.aov(t, m, periods, pdts, 10))
        got = calc_sharded(compute, ts, ms, rank, world)
        want = O.aov(ts, ms, periods, pdts, 10)
        ok = all(np.array_equal(g, w) for g, w in zip(got, want))
        mx = max_over_ranks(1.0 + rank)
        q.put((rank, ok, mx))
    finally:
        dist.destroy_process_group()


def test_sharded_calc_gloo_world2(oracle):  # fixture: oracle built before the ranks spawn
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, mx in res:
        assert ok, f"rank {rank} gathered results differ from the single-process oracle"
        assert mx == pytest.approx(2.0)
