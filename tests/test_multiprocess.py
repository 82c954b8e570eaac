"""Replica (weak-scaling) bookkeeping of bench.py across ranks, on CPU with gloo (world size 2).

The SIMPLE path does not shard (single-rank reference, GSV1:2939), so N GPUs run N independent
replicas; the only cross-rank step is the max over ranks of the timed region."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # each replica reports its own device time and e2e time; rank 1 is slower
    mine = [1.0 + rank, 2.0 - rank * 0.5]
    got = bench.max_over_ranks(mine, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, bench.replica_throughput(world, 1000, 10, got[0])))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, thr in res:
        assert got == [2.0, 2.0]          # max over ranks of [1, 2] and [2, 1.5]
        assert thr == pytest.approx(2 * 1000 * 10 / 2.0)


def test_single_rank_passthrough():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert bench.replica_throughput(1, 970480, 10, 0.17) == pytest.approx(970480 * 10 / 0.17)
