"""Benchmark: served FP32 vs plain FP64 FMM on the mixed serving stream.

Metric: FMM points/s and p99 latency of the served FP32 form against the
plain FP64 GPU form, at relative-L2 error <= 1e-6 against the FP64 direct sum.

Workload (`--workload stream`, the default): the mixed serving stream --
requests with N log-uniform in [1e3, 3e5] sources, half Laplace (order 14)
and half Helmholtz with k ~ U[1, 30] (per-level orders max(14, kw rule)),
sources uniform in the cube or on the r = 0.45 sphere (fair coin), N(0,1)
strengths (complex for Helmholtz), targets = sources, depth for about 64
points per leaf; seeded synthetic requests (the reference names no
dataset).  One step = one batch of SERVE_BATCH requests.

* `value`: the served form (SERVE_SLOTS solves at once, FP32 wherever the
  FP32 range rule admits a request, FP64 expansions with an FP32 near field
  otherwise, boxes without targets skipped) on batches whose inputs and outputs are already in device memory
  (requests submitted with device arrays); points/s = sources of the batch /
  the batch's span from the first submission to the last completion (CUDA
  events, max over ranks).  W untimed batches, then K timed ones.
* `e2e`: the same served batches through the public API with host arrays:
  the host->device copies of every request's inputs and the device->host
  copies of its fields are inside the timed span.
* `plain_fp64`: the plain form (one FP64 solve at a time, every box, the
  reference's point order) on the same batches, device-resident and host;
  `plain_fp64_skip_empty`: the same with boxes without targets skipped, so
  that the served form's gain from serving and FP32 shows apart from the
  empty-box savings.  `served_over_plain` is value / plain value.
* latency: Poisson arrivals at 30/50/70/90% of each arm's own batch
  throughput (host arrays) to one warmed server per arm, the loads one
  after another, p50 / p99 per load, and per load the p99 and maximum of
  each request's queue wait, host issue and device completion; the top-level
  `served_p50_s` / `served_p99_s` / `plain_p50_s` / `plain_p99_s` are at 70%.
* accuracy: the served fields of sampled requests against the FP64 GPU
  direct sum (itself pinned to the reference's direct sums).
* `roofline`: the stream's dominant kernel, the FP32 Helmholtz tile M2L
  (23% of the stream's device time in profiles/launches_serving_stream_48.md)
  on an order-14 level (1e5 points, k = 10, level 4): algorithmic FLOPs of
  the dense level's list-4 pairs / event time, against the FP32 FMA peak
  measured live on the GPU (`wbfmm_b200_fp32_fma_peak`), `traffic` from the
  committed ncu capture of the same launch.  `roofline_p2p`: the FP32 near
  field (k_p2p, the next kernel, 18%) on a 2e5-point Helmholtz cube, exact
  pair count; `roofline_m2l_laplace`: the Laplace tile M2L on an order-14
  level (3e5 points, level 5).
* `cpu_baseline` and `--impl reference`: the reference's own CPU FMM
  (oracle/_ref, the unmodified reference sources, M2L on up to 16 threads)
  run request by request on a bounded sample of the stream.
* `cube_c2`: the 1e6-point Helmholtz cube (k = 8, depth 6) solved once per
  step by the FP32 and FP64 forms, and through the C ABI with host buffers.

The other `--workload` values (cube, laplace_c1, sphere_c3, clusters_c5)
measure single solves of those configurations as the headline instead.

Multi-GPU: one process per GPU (torchrun), independent replicas (weak
scaling, no collective on the data path); spans are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FMM points/s + p99 latency: served FP32 vs plain FP64 GPU at rel-L2 err<=1e-6"
STREAM_WORKLOAD = ("serving_stream_N_loguniform_1e3_3e5_half_laplace_p14_half_helmholtz_"
                   "k1_30_cube_or_sphere_targets_eq_sources")
CUBE_WORKLOAD = "helmholtz_cube_1e6_k8_depth6"
SERVE_SLOTS = 6
SERVE_BATCH = 256
SERVE_LATENCY_REQUESTS = 256
SERVE_LOADS = (0.3, 0.5, 0.7, 0.9)
# the CPU reference's sample of the stream: the first requests of the first
# timed batch with at most this many sources, this many of them
CPU_SAMPLE_MAX_N = 20_000
CPU_SAMPLE_REQUESTS = 12
TILE_PROFILE = os.path.join(ROOT, "profiles", "k_m2l_tiles_laplace_3e5_p14_level5.md")


# ---------------------------------------------------------------- helpers
def list4_pairs(depth: int) -> list[int]:
    """Number of (target, list-4 source) pairs per level of a dense tree."""
    out = [0] * (depth + 1)
    for lv in range(2, depth + 1):
        n = 1 << lv
        i = np.arange(n)
        i0 = i - i % 2
        i1 = np.minimum(i0 + 3, n - 1)
        lo = np.where(i0 > 0, i0 - 2, i0)
        span = i1 - lo + 1                              # parent-neighbour extent
        near = np.minimum(i + 1, n - 1) - np.maximum(i - 1, 0) + 1
        tot = (span[:, None, None] * span[None, :, None] * span[None, None, :]).sum()
        nr = (near[:, None, None] * near[None, :, None] * near[None, None, :]).sum()
        out[lv] = int(tot - nr)
    return out


def list4_pairs_at(xt, x0, D, level: int, xs=None) -> int:
    """(target box, list-4 source box) pairs of the boxes at `level` that hold
    one of the points xt, counting only source boxes that hold one of the
    points xs when given (the M2L work of a skip_empty solve, whose kernels
    skip empty source boxes)."""
    n = 1 << level

    def boxes(pts):
        ijk = np.floor((np.asarray(pts) - np.asarray(x0)) / (D / n)).astype(np.int64)
        return np.unique(np.clip(ijk, 0, n - 1), axis=0)

    ijk = boxes(xt)
    i0 = ijk - ijk % 2
    i1 = np.minimum(i0 + 3, n - 1)
    lo = np.where(i0 > 0, i0 - 2, i0)
    nlo = np.maximum(ijk - 1, 0)
    nhi = np.minimum(ijk + 1, n - 1)
    if xs is None:
        span = i1 - lo + 1
        near = nhi - nlo + 1
        return int((span.prod(axis=1) - near.prod(axis=1)).sum())
    # occupied source boxes counted over a box range by a summed-volume table
    occ = np.zeros((n + 1, n + 1, n + 1), dtype=np.int32)
    sb = boxes(xs)
    occ[sb[:, 0] + 1, sb[:, 1] + 1, sb[:, 2] + 1] = 1
    occ = occ.cumsum(0).cumsum(1).cumsum(2)

    def count(a, b):   # boxes in [a, b] per row, inclusive
        x0_, y0_, z0_ = a[:, 0], a[:, 1], a[:, 2]
        x1_, y1_, z1_ = b[:, 0] + 1, b[:, 1] + 1, b[:, 2] + 1
        return (occ[x1_, y1_, z1_] - occ[x0_, y1_, z1_] - occ[x1_, y0_, z1_] - occ[x1_, y1_, z0_]
                + occ[x0_, y0_, z1_] + occ[x0_, y1_, z0_] + occ[x1_, y0_, z0_]
                - occ[x0_, y0_, z0_]).astype(np.int64)

    return int((count(lo, i1) - count(nlo, nhi)).sum())


def lap_flops_per_pair(p: int) -> int:
    """Algorithmic FLOPs of one Laplace rotate/coaxial/rotate-back shift on
    half vectors: 2*2*R(p) + 2*X_L(p), X_L(p) = (p+1)^2 + 2 sum_m (p+1-m)^2."""
    R = (p + 1) * (2 * p + 1) * (2 * p + 3) // 3
    XL = (p + 1) ** 2 + 2 * sum((p + 1 - m) ** 2 for m in range(1, p + 1))
    return 2 * 2 * R + 2 * XL


def helm_flops_per_pair(p: int) -> int:
    """Algorithmic FLOPs of one Helmholtz rotate/coaxial/rotate-back shift:
    2*4*R(p) + 8*X(p), R(p) = sum (2n+1)^2, X(p) = coaxial MACs."""
    R = (p + 1) * (2 * p + 1) * (2 * p + 3) // 3
    X = (p + 1) ** 2 + p * (p + 1) ** 2 - p * (p + 1) * (p + 2) // 3
    return 2 * 4 * R + 8 * X


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for s in self.samples for n, v in zip(names, s[5:9])
                          if v.strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------- reference (CPU)
def reference_sample(scale: int = 2, seed: int = 2):
    """Bounded sample of the workload for the CPU reference: the same point
    density, k, box widths and per-level orders, in a sub-cube of 1/scale^3
    of the volume (125,000 points for scale 2, depth 6 - log2(scale))."""
    from wbfmm_b200 import workloads as W
    n = 1_000_000 // scale ** 3
    depth = 6 - int(round(math.log2(scale)))
    rng = np.random.default_rng(seed)
    h = 0.5 / scale
    xs = rng.uniform(-h, h, size=(n, 3))
    q = rng.standard_normal(2 * n)
    p = W.Problem("helmholtz_subcube", W.HELMHOLTZ, depth, [0] * (depth + 1),
                  [0] * (depth + 1), 8.0, xs, q, xs, targets_are_sources=True)
    p.x0, p.D = W.fit_box(xs)
    for lv in range(1, depth + 1):
        o = W.helmholtz_order(8.0, p.D / 2 ** lv)
        p.order_s[lv] = p.order_r[lv] = o
    return p


def run_reference_step(p, nthreads):
    from oracle.oracle_api import Reference
    R = Reference()
    t0 = time.perf_counter()
    R.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs, p.q, p.xt,
          k=p.k, pot=True, grad=True, nthreads=nthreads)
    return time.perf_counter() - t0




# ------------------------------------------------------------ workloads
# name -> (builder, accuracy subsample size and seed, skip_empty, label)
def workload(args, rank):
    """The problem of --workload: the benchmark's configurations (seeded,
    synthetic; the reference names no dataset)."""
    from wbfmm_b200 import workloads as W
    w = args.workload
    if w == "cube":
        p = W.helmholtz_cube(args.points, k=8.0, depth=args.depth or 6, seed=2 + rank)
        return p, 10_000, 102, False, CUBE_WORKLOAD
    if w == "laplace_c1":
        p = W.laplace_cube(20_000, 20_000, depth=4, order=12, seed=1 + rank)
        return p, 20_000, 101, False, "laplace_cube_2e4_separate_targets_depth4_p12"
    if w == "sphere_c3":
        # per-level order p = kw + 1.8*6^(2/3)*(kw)^(1/3), floor 6, unclamped
        p = W.helmholtz_sphere(2_000_000, 500_000, k=40.0, depth=7, seed=3 + rank, hi=None)
        return p, 10_000, 103, True, "helmholtz_sphere_2e6_half_dipoles_5e5_targets_k40_depth7"
    if w == "clusters_c5":
        d = args.depth or 8
        p = W.laplace_clusters(16_000_000, depth=d, order=10, seed=5 + rank)
        return p, 20_000, 105, True, f"laplace_8_gaussian_clusters_1.6e7_depth{d}_p10"
    raise SystemExit(f"unknown workload {w}")


# ------------------------------------------------------ profiling cases
# Small, fixed workloads for profiling single kernels of the engine
# (`python bench.py --profile-case <case>`): each builds one solve, runs it
# once (warm-up: tables, buffers), then launches the stage it is named for
# once more on its own, so that a profiler filtering on that kernel's name
# with one or two captured launches sees the steady-state launch.
PROFILE_CASES = """

  m2l_tiles_laplace_p14     Laplace, 3e5 uniform points, depth 5, order 14,
                            FP32: M2L of level 5 (offset-major tile kernel)
  m2l_tiles_helmholtz_p14   Helmholtz k = 10, 1e5 points, depth 4, orders
                            max(14, kw rule), FP32: M2L of level 4
  m2l_lanes_helmholtz_p6    Helmholtz k = 8, 1e6 points, depth 6, the
                            benchmark's orders, FP32: M2L of level 6
                            (lane-per-pair kernel)
  m2l_lanes_laplace_clusters_p10
                            Laplace, 2e6 points in 8 Gaussian clusters,
                            depth 7, order 10, skip_empty, FP32: M2L of
                            level 7 (lane kernel on target lists)
  m2l_tc_laplace_p14        as m2l_tiles_laplace_p14 on the tensor cores
                            (M2L mode 4: tcgen05 3xTF32)
  p2p_helmholtz             Helmholtz k = 10, 2e5 points, depth 4, FP32:
                            evaluation (L2P + P2P)
  target_bases_helmholtz    Helmholtz k = 10, 2e5 points, depth 4, FP64:
                            potential from precomputed target bases
  served_stream             48 requests of the serving stream through a
                            1-slot server, FP32 where the range rule admits
                            the request, skip_empty and leaf_order (launch
                            lists of a served mix)
"""


def _solve_then(p, precision, stage, skip_empty=False):
    from wbfmm_b200 import engine
    cfg = engine.SolverConfig.from_problem(p, precision, skip_empty=skip_empty)
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs, p.normals).set_strengths(p.q, p.dipoles).set_targets(p.xt).run()
        stage(s)
        s.synchronize()


def _cube(problem, n, depth, order, k=0.0, seed=1):
    from wbfmm_b200 import engine, workloads as W
    rng = np.random.default_rng(seed)
    p = W.serve_request(rng, n, problem == engine.HELMHOLTZ, k, False)
    p.depth = depth
    p.order_s = [0] * (depth + 1)
    for lv in range(1, depth + 1):
        p.order_s[lv] = (W.helmholtz_order(k, p.D / 2 ** lv, lo=order, hi=60)
                         if problem == engine.HELMHOLTZ else order)
    p.order_r = list(p.order_s)
    return p


def profile_case(case: str) -> None:
    from wbfmm_b200 import engine, workloads as W
    if case == "m2l_tiles_laplace_p14":
        p = _cube(engine.LAPLACE, 300_000, 5, 14)
        _solve_then(p, engine.FP32, lambda s: s.m2l(5))
    elif case == "m2l_tc_laplace_p14":
        p = _cube(engine.LAPLACE, 300_000, 5, 14)

        def tc(s):
            s.set_m2l_kernel(4)
            s.m2l(5)
        _solve_then(p, engine.FP32, tc)
    elif case == "target_bases_helmholtz":
        p = _cube(engine.HELMHOLTZ, 200_000, 4, 8, k=10.0)
        _solve_then(p, engine.FP64, lambda s: s.target_bases().evaluate_bases())
    elif case == "m2l_tiles_helmholtz_p14":
        p = _cube(engine.HELMHOLTZ, 100_000, 4, 14, k=10.0)
        _solve_then(p, engine.FP32, lambda s: s.m2l(4))
    elif case == "m2l_lanes_helmholtz_p6":
        p = W.helmholtz_cube(1_000_000, k=8.0, depth=6, seed=2)
        _solve_then(p, engine.FP32, lambda s: s.m2l(6))
    elif case == "m2l_lanes_laplace_clusters_p10":
        p = W.laplace_clusters(2_000_000, depth=7, order=10, seed=5)
        _solve_then(p, engine.FP32, lambda s: s.m2l(7), skip_empty=True)
    elif case == "p2p_helmholtz":
        p = _cube(engine.HELMHOLTZ, 200_000, 4, 8, k=10.0)
        _solve_then(p, engine.FP32, lambda s: s.evaluate())
    elif case == "served_stream":
        reqs = list(W.serving_stream(48, seed=4))
        with engine.Server(slots=1) as srv:
            tickets = [srv.submit(p, engine.FP32 if engine.fp32_range_ok(engine.SolverConfig.from_problem(p))
                                  else engine.FP64, skip_empty=True, leaf_order=True)
                       for p in reqs]
            srv.drain()
            for t in tickets:
                srv.wait(t)
    else:
        raise SystemExit(f"unknown profiling case {case!r}; see PROFILE_CASES")



def stream_requests(args, rank):
    """The stream's requests for one rank: W warm-up batches, K timed
    batches, and the latency run's requests (seeded per rank)."""
    from wbfmm_b200 import workloads as W
    nw, nb = max(1, args.warmup), max(1, args.steps)
    gen = W.serving_stream(SERVE_BATCH * (nw + nb) + SERVE_LATENCY_REQUESTS, seed=4 + 1000 * rank)
    warm = [[next(gen) for _ in range(SERVE_BATCH)] for _ in range(nw)]
    batches = [[next(gen) for _ in range(SERVE_BATCH)] for _ in range(nb)]
    lat = [next(gen) for _ in range(SERVE_LATENCY_REQUESTS)]
    return warm, batches, lat


def stream_cpu_sample(rank=0):
    """The CPU reference's bounded sample of the stream: in stream order, the
    first CPU_SAMPLE_REQUESTS requests of the first timed batch (the same
    requests whatever the step counts) with at most CPU_SAMPLE_MAX_N sources.
    The reference's points/s falls with the request size (deeper trees, more
    M2L pairs per point), so leaving the larger requests out favours the
    reference."""
    from wbfmm_b200 import workloads as W
    gen = W.serving_stream(SERVE_BATCH * 2, seed=4 + 1000 * rank)
    reqs = [next(gen) for _ in range(SERVE_BATCH * 2)][SERVE_BATCH:]   # a batch after one warm-up
    out = [p for p in reqs if p.ns <= CPU_SAMPLE_MAX_N][:CPU_SAMPLE_REQUESTS]
    return out


def stream_config(ws):
    return {"workload": STREAM_WORKLOAD, "global_batch": ws * SERVE_BATCH, "seq_len": 0,
            "parallelism": f"replicas{ws}", "requests_per_step_per_gpu": SERVE_BATCH,
            "l2": "each step's inputs (about 0.5 GB per batch) exceed the 126 MB L2"}


def run_reference_requests(reqs, nthreads):
    """Seconds of the reference's own CPU FMM over the requests, one after
    another, as its drivers run a solve (tree, operators, passes, potential
    and gradient evaluation)."""
    from oracle.oracle_api import Reference
    R = Reference()
    t0 = time.perf_counter()
    for p in reqs:
        R.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs, p.q, p.xt,
              k=p.k, pot=True, grad=True, nthreads=nthreads)
    return time.perf_counter() - t0


def cpu_sample_text(reqs):
    nh = sum(p.problem == 2 for p in reqs)
    return (f"{len(reqs)} requests of the stream ({nh} Helmholtz, {len(reqs) - nh} Laplace; "
            f"{sum(p.ns for p in reqs)} sources; the first {CPU_SAMPLE_REQUESTS} of a batch "
            f"with N <= {CPU_SAMPLE_MAX_N}), one after another; reference FMM with M2L on "
            "GThreads (other stages serial), potential and gradient")


def reference_arm(args, ws, rank):
    """The reference's own CPU implementation (oracle/_ref) on the host
    cores, on this arm's workload, metric and config; rank 0 only."""
    if rank != 0:
        return
    from oracle.oracle_api import have_reference
    stream = args.workload == "stream"
    cfgd = stream_config(ws) if stream else {"workload": CUBE_WORKLOAD, "global_batch": ws * 1_000_000,
                                            "seq_len": 0, "parallelism": f"replicas{ws}"}
    if not have_reference():
        print(json.dumps({"impl": "reference", "metric": METRIC,
                          "unavailable": "oracle/_ref/libwbfmm_ref.so was not built"}))
        return
    nthreads = min(os.cpu_count() or 1, 16)
    if stream:
        reqs = stream_cpu_sample()
        points = sum(p.points for p in reqs)
        sample = cpu_sample_text(reqs)

        def step():
            return run_reference_requests(reqs, nthreads)
    else:
        rp = reference_sample(2)
        points = rp.points
        sample = (f"{rp.ns} points in a 1/8-volume sub-cube of the workload, depth {rp.depth}, "
                  f"orders {rp.order_s[1:]}, same density/k/box widths; reference FMM with M2L "
                  "on GThreads (others serial)")

        def step():
            return run_reference_step(rp, nthreads)
    for _ in range(args.warmup):
        step()
    times = [step() for _ in range(max(1, args.steps))]
    t = float(np.mean(times))
    v = points / t
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s",
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfgd,
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": nthreads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


# ----------------------------------------------------- served stream
def request_bytes(p):
    """(input bytes, output bytes) of a request: sources (+ normals), their
    strengths (+ dipole strengths), targets when they are not the sources;
    potential and gradient in FP64."""
    w = 2 if p.problem == 2 else 1
    nin = 24 * p.ns + 8 * w * p.ns
    if p.normals is not None:
        nin += 24 * p.ns + 8 * w * p.ns
    if not p.targets_are_sources:
        nin += 24 * p.nt
    return nin, 8 * 4 * w * p.nt


def served_section(args, ws, rank, local):
    """Served FP32 vs plain FP64 on batches of the mixed serving stream, with
    device-resident requests (value) and host arrays (e2e)."""
    import torch

    from wbfmm_b200 import engine, workloads as W

    dev = torch.device("cuda", local)
    marker = torch.cuda.Stream(dev)          # span events (the slots run their own streams)
    warm, batches, lat_reqs = stream_requests(args, rank)

    def on_dev(p):
        w = 2 if p.problem == W.HELMHOLTZ else 1

        def t(a):
            return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)

        return {"xs": t(p.xs), "q": t(p.q), "normals": t(p.normals), "dipoles": t(p.dipoles),
                "xt": None if p.targets_are_sources else t(p.xt),
                "pot": torch.empty(w * p.nt, dtype=torch.float64, device=dev),
                "grad": torch.empty(3 * w * p.nt, dtype=torch.float64, device=dev)}

    # device copies of every batch's inputs (and room for its fields), made
    # before any timing
    dev_warm = [[on_dev(p) for p in b] for b in warm]
    dev_batches = [[on_dev(p) for p in b] for b in batches]
    torch.cuda.synchronize(dev)

    def served_prec(p):
        ok = engine.fp32_range_ok(engine.SolverConfig.from_problem(p))
        return engine.FP32 if ok else engine.FP64
    # the served form runs the requests that stay in FP64 with their near
    # field in FP32 (FP64 expansions and L2P; near_fp32)
    served_prec.near32 = True

    def near32(precf, p):
        return bool(getattr(precf, "near32", False)) and precf(p) == engine.FP64

    def plain_prec(p):
        return engine.FP64

    def run_batch(srv, batch, dbatch, precf, skip, keep=0):
        dist_barrier(ws)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = srv.stats()["kernel_launches"]
        e0.record(marker)
        tk = [srv.submit(p, precf(p), skip_empty=skip, leaf_order=skip,
                         device=d if dbatch is not None else None, near_fp32=near32(precf, p))
              for p, d in zip(batch, dbatch if dbatch is not None else [None] * len(batch))]
        srv.drain()
        e1.record(marker)
        e1.synchronize()
        span = e0.elapsed_time(e1) * 1e-3
        T = np.array([srv.times(t) for t in tk])
        kept = []
        for t in tk[:keep]:
            pot, grad = srv.wait(t)
            kept.append((pot.cpu().numpy() if hasattr(pot, "cpu") else pot.copy(),
                         grad.cpu().numpy() if hasattr(grad, "cpu") else grad.copy()))
        for t in tk:
            srv.forget(t)
        return (dist_max(span, ws), kept, srv.stats()["kernel_launches"] - l0,
                float(np.mean(T[:, 2] - T[:, 1])), float(np.mean(T[:, 3] - T[:, 2])))

    def run_arm(name, slots, precf, skip, device, keep=0):
        # a batch is submitted at once: the served form's slots take its
        # largest requests first (largest-first order); one slot runs the
        # batch's solves one after another whatever the order
        with engine.Server(slots=slots, largest_first=slots > 1) as srv:
            for b, d in zip(warm, dev_warm):
                run_batch(srv, b, d if device else None, precf, skip)
            spans, launches, issue, wait = [], [], [], []
            kept = None
            with ClockSampler(local) as clk:
                for i, (b, d) in enumerate(zip(batches, dev_batches)):
                    span, k, nl, ti, tw = run_batch(srv, b, d if device else None, precf, skip,
                                                    keep=keep if i == 0 else 0)
                    spans.append(span)
                    launches.append(nl)
                    issue.append(ti)
                    wait.append(tw)
                    if k:
                        kept = k
            pts = sum(p.points for b in batches for p in b)
            return {"points_per_s": ws * pts / sum(spans), "seconds": sum(spans),
                    "ms_per_step": 1e3 * float(np.mean(spans)), "step_ms": [1e3 * s for s in spans],
                    "requests": len(batches) * SERVE_BATCH, "slots": slots, "skip_empty": skip,
                    "order": "largest first" if slots > 1 else "arrival",
                    "inputs": "device" if device else "host",
                    "kernel_launches_per_step": int(np.mean(launches)),
                    "host_issue_ms_per_request": 1e3 * float(np.mean(issue)),
                    "device_wait_ms_per_request": 1e3 * float(np.mean(wait)),
                    "clocks": clk.summary(), "stats": srv.stats()}, kept

    out = {}
    served_dev, _ = run_arm("served", SERVE_SLOTS, served_prec, True, True)
    served_host, kept = run_arm("served", SERVE_SLOTS, served_prec, True, False, keep=8)
    plain_dev, _ = run_arm("plain", 1, plain_prec, False, True)
    plain_host, _ = run_arm("plain", 1, plain_prec, False, False)
    plain_skip, _ = run_arm("plain_skip", 1, plain_prec, True, True)
    out["served_fp32"] = {"device": served_dev, "host": served_host}
    out["plain_fp64"] = {"device": plain_dev, "host": plain_host}
    out["plain_fp64_skip_empty"] = {"device": plain_skip}

    # latency under Poisson arrivals at fractions of each arm's own
    # throughput (host arrays, as a caller submits)
    mean_pts = np.mean([p.points for b in batches for p in b])

    def run_latency(srv, precf, skip, rate, seed):
        arr = W.poisson_arrivals(len(lat_reqs), rate, seed=seed + rank)
        base = srv.clock() + 0.02
        tk = [srv.submit(p, precf(p), arrival=base + a, skip_empty=skip, leaf_order=skip,
                         near_fp32=near32(precf, p))
              for p, a in zip(lat_reqs, arr)]
        srv.drain()
        T = np.array([srv.times(t) for t in tk])
        for t in tk:
            srv.forget(t)
        lat = T[:, 3] - T[:, 0]
        # where the time went: waiting for a slot (arrival -> start), the
        # slot issuing the solve (start -> queued: staging and launches on
        # the host), and the device finishing it (queued -> end)
        parts = {"queue_wait": T[:, 1] - T[:, 0], "host_issue": T[:, 2] - T[:, 1],
                 "completion": T[:, 3] - T[:, 2]}
        return {"offered_requests_per_s": float(rate),
                "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "mean_s": float(lat.mean()),
                "parts_p99_s": {k: float(np.percentile(v, 99)) for k, v in parts.items()},
                "parts_max_s": {k: float(v.max()) for k, v in parts.items()},
                "achieved_points_per_s": float(sum(p.points for p in lat_reqs) /
                                               (T[:, 3].max() - base))}

    # one long-running server per arm, warmed once (pools, tables, kernels),
    # sees the loads one after another (each drained before the next).  The
    # warm-up runs every warm-up batch: a slot builds its FP64 solver at the
    # first FP64 request it meets (a few percent of the stream), and one
    # batch over six slots leaves some without one, a first-use cost (tens
    # of ms of host issue) that would otherwise land in the first timed load
    latency = {}
    for name, slots, precf, skip, thr in (
            ("served_fp32", SERVE_SLOTS, served_prec, True, served_host["points_per_s"]),
            ("plain_fp64", 1, plain_prec, False, plain_host["points_per_s"])):
        latency[name] = {}
        with engine.Server(slots=slots) as srv:
            for b in warm:                                 # steady state
                run_batch(srv, b, None, precf, skip)
            for load in SERVE_LOADS:
                rate = load * thr / ws / mean_pts
                latency[name][f"{int(load * 100)}%"] = run_latency(srv, precf, skip, rate,
                                                                   104 + int(load * 100))
    out["latency"] = latency

    # accuracy of served fields against the FP64 direct sum
    worst, checked = 0.0, []
    for p, (pot, grad) in zip(batches[0][:8], kept or []):
        idx = W.subsample(105, p.ns, 1000)
        dpot, dgrad = engine.direct(p.problem, p.xs, p.q, p.xs[idx], k=p.k)
        w = 2 if p.problem == W.HELMHOLTZ else 1
        ep = engine.error_norms(pot.reshape(p.ns, w)[idx].ravel(), dpot)[0]
        eg = engine.error_norms(grad.reshape(p.ns, 3 * w)[idx].ravel(), dgrad)[0]
        worst = max(worst, ep, eg)
        checked.append({"n": p.ns, "problem": "helmholtz" if p.problem == W.HELMHOLTZ else "laplace",
                        "k": p.k, "fp32": served_prec(p) == engine.FP32,
                        "pot_rel_l2": ep, "grad_rel_l2": eg})
    out["accuracy"] = {"max_rel_l2": worst, "tolerance": 1e-6, "requests": checked,
                       "reference": "FP64 GPU direct sum on 1000 targets per request"}
    out["fp32_fraction"] = float(np.mean([served_prec(p) == engine.FP32
                                          for b in batches for p in b]))
    nin = sum(request_bytes(p)[0] for b in batches for p in b) // len(batches)
    nout = sum(request_bytes(p)[1] for b in batches for p in b) // len(batches)
    out["bytes_per_step"] = {"h2d": int(nin), "d2h": int(nout)}
    return out


# ------------------------------------------------- single-solve workloads
def single_solve_section(args, ws, rank, local, p, n_acc, acc_seed, skip_empty, label, steps):
    """One workload solved once per step by the FP32 and FP64 forms from
    device-resident inputs (tree, FP64 tables, passes, evaluation, queued
    with deferred checks), and by the FP32 form through the C ABI with pinned
    host buffers (e2e)."""
    import torch

    from wbfmm_b200 import engine, workloads as W

    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)     # the solvers' stream; events on it
    helm = p.problem == W.HELMHOLTZ
    w = 2 if helm else 1
    ns, nt = p.ns, p.nt
    field = engine.POTENTIAL | engine.GRADIENT

    def dev_arr(a):
        return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    xs_d, q_d = dev_arr(p.xs), dev_arr(p.q)
    nrm_d, dip_d = dev_arr(p.normals), dev_arr(p.dipoles)
    xt_d = xs_d if p.targets_are_sources else dev_arr(p.xt)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    sparse = bool(getattr(args, "sparse", False))

    def make(precision):
        # the FP32 form sorts the sources by leaf box only; the plain FP64
        # form on full keys, as the reference
        cfg = engine.SolverConfig.from_problem(p, precision, field, skip_empty,
                                               leaf_order=precision == engine.FP32,
                                               sparse=sparse)
        s = engine.Solver(cfg, stream=stream.cuda_stream)
        s.set_deferred_checks(True)     # no host wait inside a solve
        return s

    def step(s):
        s.set_sources(xs_d, nrm_d, on_device=True)
        s.set_strengths(q_d, dip_d, on_device=True)
        s.set_targets(xt_d, on_device=True)
        s.invalidate_operators()
        s.run_async()

    results = {}
    for name, prec in (("fp64", engine.FP64), ("fp32", engine.FP32)):
        s = make(prec)
        for _ in range(max(3, args.warmup)):
            step(s)
        s.wait()
        torch.cuda.synchronize(dev)
        l0 = s.kernel_launches()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        dist_barrier(ws)
        torch.cuda.synchronize(dev)
        with ClockSampler(local) as clk:
            for i in range(steps):
                with torch.cuda.stream(stream):
                    flush.zero_()                   # L2 flush between steps
                ev[i][0].record(stream)
                step(s)
                ev[i][1].record(stream)
            torch.cuda.synchronize(dev)
        s.wait()                                    # deferred checks of the last step
        dist_barrier(ws)
        step_ms = [a.elapsed_time(b) for a, b in ev]
        ms = dist_max(float(np.mean(step_ms)), ws)
        launches = (s.kernel_launches() - l0) // steps
        stages = s.stage_times()
        m2l_ms = {}
        for lv in range(2, p.depth + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.zero_()
            a.record(stream)
            s.m2l(lv)
            b.record(stream)
            torch.cuda.synchronize(dev)
            m2l_ms[lv] = a.elapsed_time(b)
        pot, grad = s.field()
        results[name] = dict(ms=ms, step_ms=step_ms, launches=launches, stages=stages,
                             m2l_ms=m2l_ms, pot=pot, grad=grad, clocks=clk.summary(),
                             coef_bytes=s.coefficient_storage(0)[1])
        if name == "fp64":
            s.close()
            torch.cuda.synchronize(dev)
        else:
            results[name]["solver"] = s

    # e2e through the C ABI with pinned host buffers (FP32 form)
    def pinned(a):
        return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).pin_memory()

    xs_h, q_h, nrm_h, dip_h = pinned(p.xs), pinned(p.q), pinned(p.normals), pinned(p.dipoles)
    xt_h = xs_h if p.targets_are_sources else pinned(p.xt)
    pot_h = torch.empty(w * nt, dtype=torch.float64).pin_memory()
    grad_h = torch.empty(3 * w * nt, dtype=torch.float64).pin_memory()
    s = results["fp32"]["solver"]

    def ptr(t):
        return None if t is None else t.data_ptr()

    def e2e_step():
        s.lib.wbfmm_b200_set_sources(s.h, ns, ptr(xs_h), 3, ptr(nrm_h), 3, 0)
        s.lib.wbfmm_b200_set_strengths(s.h, ptr(q_h), w, ptr(dip_h), w, 0)
        s.lib.wbfmm_b200_set_targets(s.h, nt, ptr(xt_h), 3, 0)
        s.invalidate_operators()
        s.run_async()
        rc = s.lib.wbfmm_b200_get_field(s.h, pot_h.data_ptr(), grad_h.data_ptr(), 0)
        assert rc == 0
        s.wait()

    for _ in range(max(1, args.warmup)):
        e2e_step()
    dist_barrier(ws)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e2e_step()
    e1.record(stream)
    e1.synchronize()
    e2e_s = dist_max(e0.elapsed_time(e1) * 1e-3 / steps, ws)
    h2d = sum(t.numel() * 8 for t in (xs_h, q_h, nrm_h, dip_h) if t is not None)
    h2d += xt_h.numel() * 8     # targets are copied even when they are the sources
    e2e = {"value": ws * p.points / e2e_s, "unit": "points/s",
           "ms_per_step": e2e_s * 1e3, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int((pot_h.numel() + grad_h.numel()) * 8)}
    s.close()

    # accuracy vs the FP64 direct sum on a seeded subsample of the targets
    idx = W.subsample(acc_seed, nt, n_acc)
    dpot, dgrad = engine.direct(p.problem, p.xs, p.q, p.xt[idx], k=p.k,
                                normals=p.normals, dipoles=p.dipoles)
    acc = {"targets_checked": int(len(idx)), "norms": "wbfmm_b200_error_norms"}
    for name in ("fp64", "fp32"):
        pot = results[name]["pot"].reshape(-1, w)[idx].ravel()
        grad = results[name]["grad"].reshape(-1, 3 * w)[idx].ravel()
        pl2, pmax = engine.error_norms(pot, dpot)
        gl2, _ = engine.error_norms(grad, dgrad)
        acc[name] = {"pot_rel_l2": pl2, "grad_rel_l2": gl2, "pot_rel_max": pmax}
    f64, f32 = results["fp64"], results["fp32"]
    acc["fp32_vs_fp64"] = {
        "pot_rel_l2": engine.error_norms(f32["pot"], f64["pot"])[0],
        "grad_rel_l2": engine.error_norms(f32["grad"], f64["grad"])[0]}

    # the dominant kernel of the solve (M2L of its busiest level, FP32)
    pairs = list4_pairs(p.depth)
    lv_dom = max(f32["m2l_ms"], key=lambda lv: f32["m2l_ms"][lv])
    if skip_empty:
        pairs[lv_dom] = list4_pairs_at(p.xt, p.x0, p.D, lv_dom, p.xs)
    fpp = helm_flops_per_pair if helm else lap_flops_per_pair
    flops = pairs[lv_dom] * fpp(p.order_s[lv_dom])
    m2l = {"kernel": f"M2L level {lv_dom}, order {p.order_s[lv_dom]}, FP32",
           "ms": f32["m2l_ms"][lv_dom], "algorithmic_flops_per_launch": flops,
           "achieved_tflops": flops / (f32["m2l_ms"][lv_dom] * 1e-3) / 1e12,
           "pairs": pairs[lv_dom],
           "pairs_counted": ("list-4 pairs of the boxes that hold targets with "
                             "source boxes that hold sources"
                             if skip_empty else "all list-4 pairs of the dense level")}
    return {
        "workload": label, "points": p.points, "sources": ns, "targets": nt, "depth": p.depth,
        "orders": p.order_s[1:], "k": p.k, "skip_empty": skip_empty,
        "storage": "sparse" if sparse else "dense",
        "fp32": {"points_per_s": ws * p.points / (f32["ms"] * 1e-3), "ms_per_step": f32["ms"],
                 "step_ms": f32["step_ms"], "stages_ms": f32["stages"], "m2l_ms": f32["m2l_ms"],
                 "launches": int(f32["launches"]), "clocks": f32["clocks"],
                 "coefficient_bytes": int(f32["coef_bytes"])},
        "fp64": {"points_per_s": ws * p.points / (f64["ms"] * 1e-3), "ms_per_step": f64["ms"],
                 "step_ms": f64["step_ms"], "stages_ms": f64["stages"], "m2l_ms": f64["m2l_ms"],
                 "clocks": f64["clocks"], "coefficient_bytes": int(f64["coef_bytes"])},
        "e2e_fp32": e2e, "accuracy": acc, "dominant_m2l": m2l,
    }


# -------------------------------------------------------------- roofline
P2P_PROFILE = os.path.join(ROOT, "profiles", "k_p2p_helmholtz_2e5.md")


def tile_profile_traffic(path=None):
    """DRAM bytes (read + write) of the launch in a committed ncu capture
    (default: the tile M2L roofline case), or None."""
    try:
        text = open(path or TILE_PROFILE).read()
    except OSError:
        return None
    tot = 0.0
    scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    for key in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
        for line in text.splitlines():
            if f"`{key}`" in line:
                try:
                    val, unit = line.split("|")[2].split()
                    tot += float(val) * scale[unit]
                except (ValueError, KeyError, IndexError):
                    return None
                break
        else:
            return None
    return tot


TILE_HELM_PROFILE = os.path.join(ROOT, "profiles", "k_m2l_tiles_helmholtz_1e5_p14_level4.md")


def tile_roofline(local, helm: bool):
    """The offset-major tile M2L on a dense level at the stream's order 14,
    FP32: Helmholtz (the stream's dominant kernel) on level 4 of 1e5 points
    (k = 10, depth 4), or Laplace on level 5 of 3e5 points (depth 5);
    algorithmic FLOPs of the rotate / coaxial / rotate-back shifts per launch
    / CUDA-event launch time (L2 flushed before each), against the FP32 FMA
    peak measured here."""
    import torch

    from wbfmm_b200 import engine

    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    peak = engine.fp32_fma_peak()
    if helm:
        p, level, n = _cube(engine.HELMHOLTZ, 100_000, 4, 14, k=10.0), 4, 100_000
    else:
        p, level, n = _cube(engine.LAPLACE, 300_000, 5, 14), 5, 300_000
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    cfg = engine.SolverConfig.from_problem(p, engine.FP32)
    with engine.Solver(cfg, stream=stream.cuda_stream) as s:
        s.set_m2l_kernel(3)
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
        times = []
        for i in range(6):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.zero_()
            a.record(stream)
            s.m2l(level)
            b.record(stream)
            torch.cuda.synchronize(dev)
            if i:
                times.append(a.elapsed_time(b))
    ms = float(np.mean(times))
    order = p.order_s[level]
    fpp = helm_flops_per_pair if helm else lap_flops_per_pair
    flops = list4_pairs(p.depth)[level] * fpp(order)
    achieved = flops / (ms * 1e-3) / 1e12
    prof = TILE_HELM_PROFILE if helm else TILE_PROFILE
    name = "Helmholtz, k = 10" if helm else "Laplace"
    return {"bound": "simt",
            "kernel": f"k_m2l_tiles<float, {'Helmholtz' if helm else 'Laplace'}>: M2L of level "
                      f"{level}, order {order}, {n:,} points ({name}), depth {p.depth}",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "FP32 FMA throughput measured live (wbfmm_b200_fp32_fma_peak)",
            "traffic": tile_profile_traffic(prof),
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of the same launch, "
                              "profiles/" + os.path.basename(prof),
            "algorithmic_flops_per_launch": flops, "ms_per_launch": ms}


def p2p_pairs(s, depth):
    """(target, source) pairs of the near field with targets = sources:
    every point against the points of its leaf's 27 neighbours, less the
    self pairs (the r > 1e-6 cutoff)."""
    from wbfmm_b200 import engine
    _, bi, bn = s.tree(depth)
    n = 1 << depth
    idx = np.arange(8 ** depth, dtype=np.uint64)
    def gather(v):
        r = np.zeros(idx.shape, dtype=np.int64)
        for b in range(depth):
            r |= ((v >> np.uint64(3 * b)) & np.uint64(1)).astype(np.int64) << b
        return r
    i, j, k = gather(idx), gather(idx >> np.uint64(1)), gather(idx >> np.uint64(2))
    grid = np.zeros((n, n, n), dtype=np.int64)
    grid[i, j, k] = bn.astype(np.int64)
    pad = np.pad(grid, 1)
    nsum = sum(pad[1 + a:1 + a + n, 1 + b:1 + b + n, 1 + c:1 + c + n]
               for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1))
    return int((grid * nsum).sum() - bn.astype(np.int64).sum())


def p2p_roofline(local):
    """The FP32 near field (Helmholtz potential and gradient, 44 flops per
    pair with each MUFU operation counted once): 2e5 points, depth 4,
    k = 10; its time is the evaluation's minus the L2P's (CUDA events, L2
    flushed before each), against the FP32 FMA peak measured here."""
    import torch

    from wbfmm_b200 import engine

    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    peak = engine.fp32_fma_peak()
    p = _cube(engine.HELMHOLTZ, 200_000, 4, 8, k=10.0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    cfg = engine.SolverConfig.from_problem(p, engine.FP32)

    def timed(s):
        times = []
        for i in range(6):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.zero_()
            a.record(stream)
            s.evaluate()
            b.record(stream)
            torch.cuda.synchronize(dev)
            if i:
                times.append(a.elapsed_time(b))
        return float(np.mean(times))
    with engine.Solver(cfg, stream=stream.cuda_stream) as s:
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
        pairs = p2p_pairs(s, 4)
        both = timed(s)
        s.set_evaluation(engine.POTENTIAL | engine.GRADIENT, neighbours=False)
        l2p = timed(s)
    ms = both - l2p
    flops = pairs * 44
    achieved = flops / (ms * 1e-3) / 1e12
    return {"bound": "simt", "kernel": "k_p2p<float, Helmholtz> potential + gradient: near field "
                                       "of 200,000 points, depth 4",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "FP32 FMA throughput measured live (wbfmm_b200_fp32_fma_peak)",
            "traffic": tile_profile_traffic(P2P_PROFILE),
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of the same launch, "
                              "profiles/k_p2p_helmholtz_2e5.md",
            "pairs_per_launch": pairs, "algorithmic_flops_per_launch": flops,
            "ms_per_launch": ms, "gpairs_per_s": pairs / (ms * 1e-3) / 1e9}


# ----------------------------------------------------------- our arm
def our_arm(args, ws, rank, local):
    import torch

    from wbfmm_b200 import workloads as W

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.workload != "stream":
        p, n_acc, acc_seed, skip_empty, label = workload(args, rank)
        sec = single_solve_section(args, ws, rank, local, p, n_acc, acc_seed, skip_empty,
                                   label, args.steps)
        cpu = None
        if rank == 0 and ws == 1 and not args.no_cpu_baseline and args.workload == "cube":
            from oracle.oracle_api import have_reference
            if have_reference():
                rp = reference_sample(2)
                nthreads = min(os.cpu_count() or 1, 16)
                t = run_reference_step(rp, nthreads)
                cpu = {"value": rp.points / t, "unit": "points/s", "cores": nthreads,
                       "kind": "reference",
                       "sample": f"{rp.ns} points in a 1/8-volume sub-cube of the workload "
                                 f"(depth {rp.depth}, same density, k and box widths), one solve"}
        m = sec["dominant_m2l"]
        from wbfmm_b200 import engine
        peak = engine.fp32_fma_peak()
        line = {
            "metric": METRIC, "value": sec["fp32"]["points_per_s"], "unit": "points/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec["fp32"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": label, "global_batch": ws * p.points, "seq_len": 0,
                       "parallelism": f"replicas{ws}", "l2": "256 MiB written between steps"},
            "single_solve": sec, "e2e": sec["e2e_fp32"],
            "roofline": {"bound": "simt", "kernel": m["kernel"], "achieved": m["achieved_tflops"],
                         "peak": peak, "unit": "TFLOP/s", "frac": m["achieved_tflops"] / peak,
                         "traffic": None,
                         "peak_source": "FP32 FMA throughput measured live"},
            "cpu_baseline": cpu, "gpu_launches": sec["fp32"]["launches"],
            "clocks": sec["fp32"]["clocks"],
        }
        if rank == 0:
            print(json.dumps(line))
        return

    served = served_section(args, ws, rank, local)
    sd, sh = served["served_fp32"]["device"], served["served_fp32"]["host"]
    pd, ph = served["plain_fp64"]["device"], served["plain_fp64"]["host"]
    pskip = served["plain_fp64_skip_empty"]["device"]
    lat = served["latency"]
    cube = None
    if not args.no_cube:
        p, n_acc, acc_seed, skip_empty, label = W.helmholtz_cube(1_000_000, k=8.0, depth=6,
                                                                 seed=2 + rank), 10_000, 102, \
            False, CUBE_WORKLOAD
        cube = single_solve_section(args, ws, rank, local, p, n_acc, acc_seed, skip_empty,
                                    label, min(args.steps, 5))
        for k in ("fp32", "fp64"):
            cube[k].pop("step_ms", None)
    roofline = tile_roofline(local, helm=True)
    roofline_p2p = p2p_roofline(local)
    roofline_m2l_laplace = tile_roofline(local, helm=False)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle.oracle_api import have_reference
        if have_reference():
            reqs = stream_cpu_sample(rank)
            nthreads = min(os.cpu_count() or 1, 16)
            t = run_reference_requests(reqs, nthreads)
            cpu = {"value": sum(p.points for p in reqs) / t, "unit": "points/s",
                   "cores": nthreads, "kind": "reference", "sample": cpu_sample_text(reqs)}
    line = {
        "metric": METRIC, "value": sd["points_per_s"], "unit": "points/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sd["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": stream_config(ws),
        "served_over_plain": sd["points_per_s"] / pd["points_per_s"],
        "served_over_plain_e2e": sh["points_per_s"] / ph["points_per_s"],
        "served_over_plain_skip_empty": sd["points_per_s"] / pskip["points_per_s"],
        "served_p50_s": lat["served_fp32"]["70%"]["p50_s"],
        "served_p99_s": lat["served_fp32"]["70%"]["p99_s"],
        "plain_p50_s": lat["plain_fp64"]["70%"]["p50_s"],
        "plain_p99_s": lat["plain_fp64"]["70%"]["p99_s"],
        "served_max_rel_l2": served["accuracy"]["max_rel_l2"],
        "plain_fp64_points_per_s": pd["points_per_s"],
        "fp32_fraction": served["fp32_fraction"],
        "e2e": {"value": sh["points_per_s"], "unit": "points/s", "ms_per_step": sh["ms_per_step"],
                "h2d_bytes_per_step": ws * served["bytes_per_step"]["h2d"],
                "d2h_bytes_per_step": ws * served["bytes_per_step"]["d2h"]},
        "roofline": roofline, "roofline_p2p": roofline_p2p,
        "roofline_m2l_laplace": roofline_m2l_laplace, "cpu_baseline": cpu,
        "gpu_launches": sd["kernel_launches_per_step"], "clocks": sd["clocks"],
        "served": served, "cube_c2": cube,
    }
    if rank == 0:
        print(json.dumps(line))


def free_port() -> int:
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def torchrun_command(argv, n, port):
    """This script under torchrun with n ranks on this node (rendezvous on
    127.0.0.1), bounded by `timeout`."""
    return ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run",
            "--nnodes=1", f"--nproc-per-node={n}", "--master-addr", "127.0.0.1",
            "--master-port", str(port), os.path.abspath(__file__)] + list(argv)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=1_000_000)
    ap.add_argument("--depth", type=int, default=None,
                    help="tree depth of the cube (default 6) and clusters_c5 (default 8) workloads")
    ap.add_argument("--sparse", action="store_true",
                    help="single-solve workloads: sparse level storage (coefficients of the "
                         "groups of boxes whose parent holds points only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cube", action="store_true",
                    help="stream workload: leave out the 1e6-point cube single solves")
    ap.add_argument("--profile-case", default=None,
                    help="run one small profiling case instead of the benchmark "
                         "(see PROFILE_CASES)")
    ap.add_argument("--workload", default="stream",
                    choices=["stream", "cube", "laplace_c1", "sphere_c3", "clusters_c5"],
                    help="stream (default): the served-vs-plain serving stream; the others "
                         "measure single solves of the benchmark's further configurations")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # not under torchrun: launch one rank per GPU, as the contract's
        # launcher would
        sys.exit(subprocess.call(torchrun_command(sys.argv[1:], args.gpus, free_port())))
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            reference_arm(args, ws, rank)
        else:
            our_arm(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
