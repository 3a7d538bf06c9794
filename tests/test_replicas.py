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
        # and serves its own seeded requests of the stream
        r = next(W.serving_stream(1, seed=4 + 1000 * rank))
        cfg = bench.stream_config(ws)
        out.put((rank, t, float(p.xs[0, 0]), p.points, float(r.xs[0, 0]), cfg["global_batch"]))
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
    (r0, t0, x0, n0, s0, b0), (r1, t1, x1, n1, s1, b1) = res
    assert t0 == t1 == 11.0                          # both ranks report the slowest
    assert x0 != x1                                  # independent replicas
    assert s0 != s1                                  # and independent request streams
    assert b0 == b1 == 2 * 256                       # the job's batch counts both ranks
    # whole-job throughput: all ranks' points over the max time
    assert (n0 + n1) / t0 == 2 * n0 / 11.0


def test_bench_launches_ranks_itself():
    """bench.py --gpus N outside torchrun re-runs itself under torchrun with
    N ranks on 127.0.0.1 (the command only; no GPU here)."""
    sys.path.insert(0, ROOT)
    import bench
    cmd = bench.torchrun_command(["--gpus", "4", "--steps", "2"], 4, 29555)
    assert cmd[cmd.index("-m") + 1] == "torch.distributed.run"
    assert "--nproc-per-node=4" in cmd and "--nnodes=1" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-4:] == [os.path.join(ROOT, "bench.py"), "--gpus", "4", "--steps", "2"][-4:]
    assert cmd[0] == "timeout"
