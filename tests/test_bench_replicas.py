"""The N>1 bench path: independent replicas, time = max over ranks.  Runs two
gloo ranks on CPU (the GPU path does not shard, so no data-path collective)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    elapsed = [120.0, 150.0][rank]  # each rank's own timed region, ms
    m = bench.reduce_max(elapsed, dist)
    value = bench.replica_throughput(10, m, world)
    q.put((rank, m, value))
    dist.destroy_process_group()


def test_replica_timing_takes_max_over_ranks():
    pytest.importorskip("torch")
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, m, value in res:
        assert m == 150.0
        assert abs(value - 2 * 10 / 0.150) < 1e-9


def test_single_rank_reduce_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.5, None) == 3.5
    assert bench.replica_throughput(20, 1000.0, 1) == 20.0
