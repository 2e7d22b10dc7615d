"""The replica form of the benchmark with real solves: two ranks (a gloo
process group; both on the one device a test box has, since replicas share
nothing and none waits on another's kernels), each solving the vc_3lev_16
fixture on its own stream and timing its solves with CUDA events, then the
whole-job rate from the slowest rank (bench.replica_rate, a MAX all-reduce).
Each rank's solve is the reference's, bit for bit."""
import json
import os
import socket

import numpy as np
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
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import bench
    from conftest import golden, load_cmg
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    cmg = load_cmg()
    meta, arrays = golden("vc_3lev_16")
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
    h.fill_synthetic(meta["seed"])
    h.use_graphs(True)
    p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                         eps=meta["eps"], hang=meta["hang"])
    h.solve(p)  # warm-up: tuning and graph capture
    stream = torch.cuda.ExternalStream(h.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    a.record(stream)
    n = 3
    outs = [h.solve(p) for _ in range(n)]
    b.record(stream)
    b.synchronize()
    rate, ms = bench.replica_rate(a.elapsed_time(b), n, dist, device="cpu")
    same = all(np.array_equal(o["history"], np.array(meta["residual_history"])) for o in outs)
    same = same and all(np.array_equal(h.phi(l), arrays[f"phi{l}"]) for l in range(len(meta["boxes"])))
    q.put(json.dumps({"rank": rank, "local_ms": a.elapsed_time(b), "ms": ms, "rate": rate, "same": same}))
    h.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_two_replicas_solve_and_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [json.loads(q.get(timeout=600)) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    slowest = max(o["local_ms"] for o in out)
    for o in out:
        assert o["same"], o
        assert o["ms"] == pytest.approx(slowest)
        assert o["rate"] == pytest.approx(2 * 3 / (slowest / 1000.0))
