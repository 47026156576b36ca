"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1 run the same reduction
the NCCL ranks run on GPUs (max of the per-rank times, sum of the per-rank trial counts)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: 10 + r ms for 1000 * (r + 1) trials
        t, n = bench.aggregate_over_ranks(10.0 + rank, 1000 * (rank + 1), world, "cpu")
        out.put((rank, t, n))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_like_the_gpu_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 11.0, 3000), (1, 11.0, 3000)]


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.aggregate_over_ranks(7.5, 123, 1, "cpu") == (7.5, 123)


def _partition_rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # every rank gathers the replica indices of all ranks (the only exchange is this check)
        mine = bench.partition_replicas(256, rank, world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        t, n = bench.aggregate_over_ranks(1.0 + rank, len(mine), world, "cpu")
        out.put((rank, got, t, n))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_partition_covers_every_replica_once_over_two_gloo_ranks():
    # the 256-box (and 64-box) batches split over ranks with no exchange: the replicas of the two
    # ranks are disjoint, together all of them, and the whole-job count sums over the ranks
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partition_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, got, t, n in res:
        assert sorted(got[0] + got[1]) == list(range(256))
        assert not set(got[0]) & set(got[1])
        assert (t, n) == (2.0, 256)
    sizes = [len(bench_partition) for bench_partition in res[0][1]]
    assert max(sizes) - min(sizes) <= 1
