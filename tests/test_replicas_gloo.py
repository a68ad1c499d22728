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


def test_single_process_fallbacks():
    from vulcan.gpu import replicas as R
    assert R.shard_runs([[1], [2, 3]], 0, 1) == [0, 1]
    assert R.max_over_ranks(3.0) == 3.0
