"""The multi-GPU plumbing on two gloo ranks (CPU): runs are dealt to ranks without overlap or loss and with
balanced spectra, and the report collectives give the slowest rank's time and the job totals."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from vulcan.gpu import replicas as R
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sizes = [5000, 60000, 12000, 7000, 33000, 20000, 9000]
        runs = [list(range(n)) for n in sizes]
        mine = R.shard_runs(runs, rank, world)
        t = R.max_over_ranks(1.5 + rank)
        n = R.sum_over_ranks(sum(sizes[i] for i in mine))
        q.put((rank, mine, t, n))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_report():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [5000, 60000, 12000, 7000, 33000, 20000, 9000]
    all_runs = sorted(i for _, mine, _, _ in out for i in mine)
    assert all_runs == list(range(len(sizes)))                    # every run exactly once
    loads = [sum(sizes[i] for i in mine) for _, mine, _, _ in out]
    assert max(loads) <= sum(sizes) / 2 + max(sizes) / 2             # balanced by size
    assert all(t == 2.5 for _, _, t, _ in out)                        # the slowest rank's time
    assert all(n == sum(sizes) for _, _, _, n in out)


def _search_worker(rank, world, port, q):
    """search_runs on gloo ranks with a stand-in for Searcher.search_many (a table per run computed on the CPU)."""
    import pyarrow as pa
    import torch.distributed as dist
    from vulcan.gpu import replicas as R
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        runs = [list(range(n)) for n in (5000, 60000, 12000, 7000, 33000, 20000, 9000)]

        def fake_search_many(rs):
            return [(pa.table({"spec_idx": pa.array(r[:3]), "rank_of_searcher": pa.array([rank] * 3)}),
                     {"n": len(r)}) for r in rs]
        mine = R.search_runs(runs, fake_search_many)
        every = R.search_runs(runs, fake_search_many, gather=True)
        q.put((rank, [(i, t.column("rank_of_searcher").to_pylist(), st) for i, t, st in mine],
               [(i, t.column("rank_of_searcher").to_pylist(), st) for i, t, st in every]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_search_runs():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_search_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [5000, 60000, 12000, 7000, 33000, 20000, 9000]
    mine = {rank: m for rank, m, _ in out}
    # each rank searched only its shard, every run exactly once over the ranks, by the rank that owns it
    got = sorted(i for m in mine.values() for i, _, _ in m)
    assert got == list(range(len(sizes)))
    for rank, m in mine.items():
        assert all(who == [rank] * 3 and st["n"] == sizes[i] for i, who, st in m)
    # gathered: on both ranks all runs in run order, each from its owner
    owner = {i: rank for rank, m in mine.items() for i, _, _ in m}
    for _, _, every in out:
        assert [i for i, _, _ in every] == list(range(len(sizes)))
        assert all(who == [owner[i]] * 3 for i, who, _ in every)


def test_single_process_fallbacks():
    from vulcan.gpu import replicas as R
    assert R.shard_runs([[1], [2, 3]], 0, 1) == [0, 1]
    assert R.max_over_ranks(3.0) == 3.0
    res = R.search_runs([[1], [2, 3]], lambda rs: [(len(r), None) for r in rs])
    assert [(i, t) for i, t, _ in res] == [(0, 1), (1, 2)]
