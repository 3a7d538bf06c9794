"""Replica scaling (bench.py --gpus N): one independent solve per rank, no
data-path collective; the step time is the maximum over ranks and the value
counts every rank's points.  Exercised here with world size 2 on the gloo
backend (CPU)."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    from wbfmm_b200 import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        bench.dist_barrier(ws)
        t = bench.dist_max(10.0 + rank, ws)          # per-rank step time, max over ranks
        # each rank solves its own seeded replica of the workload
        p = W.helmholtz_cube(2000, k=8.0, depth=2, seed=2 + rank)
        out.put((rank, t, float(p.xs[0, 0]), p.points))
    finally:
        dist.destroy_process_group()


def test_replicas_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    (r0, t0, x0, n0), (r1, t1, x1, n1) = res
    assert t0 == t1 == 11.0                          # both ranks report the slowest
    assert x0 != x1                                  # independent replicas
    # whole-job throughput: all ranks' points over the max time
    assert (n0 + n1) / t0 == 2 * n0 / 11.0
