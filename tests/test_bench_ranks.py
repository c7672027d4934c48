"""bench.py's multi-rank logic on CPU: two gloo ranks (the bench's replicas
run one seeded lambda grid per rank with no collective on the data path;
the only exchange is the max-over-ranks of the timings)."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local = [1.5 + rank, 10.0 - rank]           # per-rank step time and e2e time (s)
        mx = bench.max_over_ranks(local, world, dist, "cpu")
        value = bench.weak_rate(64 * 3, world, mx[0])
        seed_sky = bench.workload(seed=7 + rank).sky.sum()
        q.put((rank, mx, value, float(seed_sky)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_weak_scale():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, value, _ in out:
        assert mx == [2.5, 10.0]                    # max over ranks, element-wise
        assert value == pytest.approx(2 * 64 * 3 / 2.5)
    assert out[0][3] != out[1][3]                   # each rank solves its own seeded grid


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.0], 1) == [3.0, 4.0]
    assert bench.weak_rate(64, 1, 2.0) == 32.0
