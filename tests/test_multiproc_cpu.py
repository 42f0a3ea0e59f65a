"""World-size-2 gloo tests of the multi-GPU host logic (run on CPU).

bench.py --gpus N runs independent replicas (one evolution per rank, no data-path
collective); the only cross-rank steps are the barrier and the max-over-ranks timing with
the summed point updates. The batched engine shards independent evolutions over ranks
with a load-balanced partition; both are checked here with two gloo ranks.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    ms = 100.0 if rank == 0 else 250.0
    pts = 1000 * (rank + 1)
    value, mx = bench.aggregate(pts, 10, ms, dist)
    from nrpy_b200.batch import partition_evolutions

    sizes = [50, 10, 40, 30, 20, 60, 5, 25]
    parts = partition_evolutions(sizes, world)
    q.put((rank, value, mx, parts))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_and_partition_gloo():
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
    res.sort()
    for rank, value, mx, parts in res:
        assert mx == 250.0
        assert value == pytest.approx((1000 + 2000) * 10 / 0.25)
    parts = res[0][3]
    assert parts == res[1][3]  # every rank derives the same partition
    assert sorted(i for p in parts for i in p) == list(range(8))
    loads = [sum([50, 10, 40, 30, 20, 60, 5, 25][i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= 60  # greedy longest-processing-time balance
