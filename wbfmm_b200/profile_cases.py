"""Small, fixed workloads for profiling single kernels of the engine.

    python -m wbfmm_b200.profile_cases <case>

Each case builds one solve, runs it once (warm-up: tables, buffers), then
launches the stage it is named for once more on its own, so that a profiler
filtering on that kernel's name with one or two captured launches sees the
steady-state launch.  Cases:

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
  p2p_helmholtz             Helmholtz k = 10, 2e5 points, depth 4, FP32:
                            evaluation (L2P + P2P)
  served_stream             48 requests of the serving stream through a
                            1-slot server, FP32 where the range rule admits
                            the request, skip_empty and leaf_order (launch
                            lists of a served mix)
"""
from __future__ import annotations

import sys

import numpy as np

from . import engine as E
from . import workloads as W


def _solve_then(p, precision, stage, skip_empty=False):
    cfg = E.SolverConfig.from_problem(p, precision, skip_empty=skip_empty)
    with E.Solver(cfg) as s:
        s.set_sources(p.xs, p.normals).set_strengths(p.q, p.dipoles).set_targets(p.xt).run()
        stage(s)
        s.synchronize()


def _cube(problem, n, depth, order, k=0.0, seed=1):
    rng = np.random.default_rng(seed)
    p = W.serve_request(rng, n, problem == E.HELMHOLTZ, k, False)
    p.depth = depth
    p.order_s = [0] * (depth + 1)
    for lv in range(1, depth + 1):
        p.order_s[lv] = (W.helmholtz_order(k, p.D / 2 ** lv, lo=order, hi=60)
                         if problem == E.HELMHOLTZ else order)
    p.order_r = list(p.order_s)
    return p


def main(case: str) -> None:
    if case == "m2l_tiles_laplace_p14":
        p = _cube(E.LAPLACE, 300_000, 5, 14)
        _solve_then(p, E.FP32, lambda s: s.m2l(5))
    elif case == "m2l_tiles_helmholtz_p14":
        p = _cube(E.HELMHOLTZ, 100_000, 4, 14, k=10.0)
        _solve_then(p, E.FP32, lambda s: s.m2l(4))
    elif case == "m2l_lanes_helmholtz_p6":
        p = W.helmholtz_cube(1_000_000, k=8.0, depth=6, seed=2)
        _solve_then(p, E.FP32, lambda s: s.m2l(6))
    elif case == "m2l_lanes_laplace_clusters_p10":
        p = W.laplace_clusters(2_000_000, depth=7, order=10, seed=5)
        _solve_then(p, E.FP32, lambda s: s.m2l(7), skip_empty=True)
    elif case == "p2p_helmholtz":
        p = _cube(E.HELMHOLTZ, 200_000, 4, 8, k=10.0)
        _solve_then(p, E.FP32, lambda s: s.evaluate())
    elif case == "served_stream":
        reqs = list(W.serving_stream(48, seed=4))
        with E.Server(slots=1) as srv:
            tickets = [srv.submit(p, E.FP32 if E.fp32_range_ok(E.SolverConfig.from_problem(p))
                                  else E.FP64, skip_empty=True, leaf_order=True)
                       for p in reqs]
            srv.drain()
            for t in tickets:
                srv.wait(t)
    else:
        raise SystemExit(f"unknown case {case!r}; see the module docstring")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "")
