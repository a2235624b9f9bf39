"""The N > 1 host paths on CPU with two gloo ranks: the cost partition of the batched replicas
(every rank computes the same split without communication; together the ranks cover each replica
once) and the max-over-ranks reduction of the benchmark's timings."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import __graft_entry__ as ge
        pd = ge.load_package()
        import bench
        specs = pd.synthetic.replica_set(64, seed=5)
        mine = pd.batch.partition_by_cost(specs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        worst = bench.max_over_ranks(world, float(10 + rank))
        out.put((rank, gathered, worst, [pd.batch.replica_cost(specs[k]) for k in mine]))
    finally:
        dist.destroy_process_group()


def test_batch_partition_and_rank_max_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # every rank computed the same partition on its own
    assert res[0][1] == res[1][1]
    parts = res[0][1]
    flat = sorted(k for part in parts for k in part)
    assert flat == list(range(64))
    loads = [sum(r[3]) for r in res]
    assert max(loads) <= 1.05 * min(loads)   # greedy longest-first split of 64 replicas
    # the timing reduction takes the slowest rank
    assert res[0][2] == res[1][2] == 11.0


def test_partition_single_rank_is_everything(pd):
    specs = pd.synthetic.replica_set(10, seed=1)
    assert pd.batch.partition_by_cost(specs, 1) == [list(range(10))]
    with pytest.raises(ValueError):
        pd.batch.partition_by_cost(specs, 0)
