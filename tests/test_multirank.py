"""The N > 1 path of bench.py on CPU: world_size-2 gloo ranks, each a replica
with its own time; the whole-job value uses the slowest rank's time on every
rank (max over ranks), and all ranks see the same numbers."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_ms = 100.0 * (rank + 1)          # rank 1 is the slow one
    value, total = bench.whole_job_value(10, local_ms, world, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, value, total))


def test_whole_job_value_is_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, value, total in res:
        assert total == pytest.approx(200.0)
        assert value == pytest.approx(10 * 2 / 0.2)


def test_single_rank_value():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    v, t = bench.whole_job_value(21, 105.0, 1)
    assert t == 105.0 and v == pytest.approx(200.0)
