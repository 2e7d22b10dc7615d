"""Multi-GPU form of the benchmark: independent replicas, one process per GPU
(replicas only: a hierarchy solve has no exchange between ranks).  The whole-job
rate is every rank's units over the slowest rank's time (a MAX all-reduce).
Checked here with world-size-2 gloo process groups on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import sys
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank r took (r + 1) * 100 ms for its 5 solves
    rate, ms = bench.replica_rate(100.0 * (rank + 1), 5, dist, device="cpu")
    q.put((rank, rate, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_rate_takes_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, ms in out:
        assert ms == 200.0                      # the slowest rank's time on every rank
        assert rate == pytest.approx(2 * 5 / 0.2)  # both ranks' solves over that time


def test_single_process_rate():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    rate, ms = bench.replica_rate(250.0, 5, None)
    assert ms == 250.0 and rate == pytest.approx(20.0)
