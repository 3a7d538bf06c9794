"""Served form: continuous batching of independent solves (serve.cu).

GPU tests: a request's fields are the same alone and inside a mixed stream;
served FP32 fields meet 1e-6 relative-L2 against the FP64 direct sum; served
FP64 fields equal the plain solver's; admission against the memory budget;
a failing request leaves the others intact.  CPU tests: the serving-stream
generator, the latency runs' arrivals and the host-side helpers (footprint,
FP32 range rule).
"""
import math

import numpy as np
import pytest

from wbfmm_b200 import engine as E
from wbfmm_b200 import workloads as W

FP32_TOL = 1e-6


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# ------------------------------------------------------------------ CPU side
def test_stream_shapes():
    reqs = list(W.serving_stream(48, seed=4, n_hi=2e4))
    assert len(reqs) == 48
    assert {p.problem for p in reqs} == {E.LAPLACE, E.HELMHOLTZ}
    for p in reqs:
        assert 1000 <= p.ns <= 20000
        assert p.targets_are_sources
        assert p.depth == max(2, round(math.log(p.ns / 64, 8)))
        if p.problem == E.LAPLACE:
            assert p.order_s[1:] == [14] * p.depth
        else:
            assert 1.0 <= p.k <= 30.0
            assert min(p.order_s[1:]) >= 14
        assert np.all(p.xs > p.x0) and np.all(p.xs < p.x0 + p.D)


def test_fp32_range_rule():
    cfg = E.SolverConfig(E.LAPLACE, 4, [0] + [14] * 4, [0] + [14] * 4, D=1.0)
    assert E.fp32_range_ok(cfg)
    cfg.order_s = cfg.order_r = [0] + [20] * 4
    assert not E.fp32_range_ok(cfg)
    hi = E.SolverConfig(E.HELMHOLTZ, 3, [0, 20, 16, 14], [0, 20, 16, 14], k=30.0, D=1.0)
    lo = E.SolverConfig(E.HELMHOLTZ, 4, [0] + [14] * 4, [0] + [14] * 4, k=1.0, D=1.0)
    assert E.fp32_range_ok(hi)
    assert not E.fp32_range_ok(lo)


def test_poisson_arrivals():
    """The latency runs' arrival times: increasing, seeded, and at the
    offered rate (mean gap 1/rate; exponential gaps, so the coefficient of
    variation is near one)."""
    a = W.poisson_arrivals(20_000, 500.0, seed=7)
    assert np.all(np.diff(a) > 0) and a[0] > 0
    assert np.array_equal(a, W.poisson_arrivals(20_000, 500.0, seed=7))
    gaps = np.diff(np.concatenate([[0.0], a]))
    assert abs(gaps.mean() * 500.0 - 1.0) < 0.03
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05


def test_footprint_grows_with_size():
    p1 = W.serve_request(np.random.default_rng(0), 2000, True, 5.0, False)
    p2 = W.serve_request(np.random.default_rng(0), 200000, True, 5.0, False)
    f1 = E.footprint(E.SolverConfig.from_problem(p1), 2000, 2000)
    f2 = E.footprint(E.SolverConfig.from_problem(p2), 200000, 200000)
    assert 0 < f1 < f2


# ------------------------------------------------------------------ GPU side
def _direct_check(p, pot, grad, m=1500, seed=5):
    idx = np.sort(np.random.default_rng(seed).choice(p.ns, size=min(m, p.ns), replace=False))
    po, go = E.direct(p.problem, p.xs, p.q, p.xs[idx], k=p.k)
    w = 2 if p.problem == E.HELMHOLTZ else 1
    return (rel(pot.reshape(p.ns, w)[idx].ravel(), po),
            rel(grad.reshape(p.ns, 3 * w)[idx].ravel(), go))


def _precision(p):
    return E.FP32 if E.fp32_range_ok(E.SolverConfig.from_problem(p)) else E.FP64


@pytest.mark.gpu
def test_same_alone_and_in_the_mix(gpu_lib):
    reqs = list(W.serving_stream(24, seed=21, n_hi=4e4))
    probe = reqs[5]
    with E.Server(slots=1) as s:
        t = s.submit(probe, _precision(probe))
        alone = [a.copy() for a in s.wait(t)]
    with E.Server(slots=8) as s:
        tickets = [s.submit(p, _precision(p)) for p in reqs]
        tickets.append(s.submit(probe, _precision(probe)))   # a second copy
        s.drain()
        for t in (tickets[5], tickets[-1]):
            mixed = s.wait(t)
            for a, b in zip(alone, mixed):
                assert rel(b, a) <= 1e-12
        st = s.stats()
        assert st["completed"] == len(reqs) + 1
        assert st["peak_solves_in_flight"] > 1


@pytest.mark.gpu
def test_served_fp32_meets_tolerance(gpu_lib):
    reqs = list(W.serving_stream(40, seed=22, n_hi=6e4))
    with E.Server(slots=8) as s:
        tickets = [(p, s.submit(p, _precision(p))) for p in reqs]
        worst = 0.0
        nfp32 = 0
        for p, t in tickets[:12]:
            pot, grad = s.wait(t)
            ep, eg = _direct_check(p, pot, grad)
            worst = max(worst, ep, eg)
            nfp32 += _precision(p) == E.FP32
        s.drain()
    assert nfp32 >= 6
    assert worst <= FP32_TOL, worst


@pytest.mark.gpu
def test_served_fp64_equals_plain(gpu_lib):
    reqs = list(W.serving_stream(6, seed=23, n_hi=3e4))
    with E.Server(slots=4) as s:
        tickets = [s.submit(p, E.FP64) for p in reqs]
        for p, t in zip(reqs, tickets):
            pot, grad = s.wait(t)
            ppot, pgrad = E.solve(p, precision=E.FP64)
            assert rel(pot, ppot) <= 1e-13 and rel(grad, pgrad) <= 1e-13


@pytest.mark.gpu
def test_admission_budget(gpu_lib):
    reqs = list(W.serving_stream(12, seed=24, n_hi=3e4))
    fps = [E.footprint(E.SolverConfig.from_problem(p, E.FP64), p.ns, p.ns) for p in reqs]
    budget = int(max(fps) * 1.5)
    with E.Server(slots=8, hbm_budget=budget) as s:
        tickets = [s.submit(p, E.FP64) for p in reqs]
        s.drain()
        st = s.stats()
        assert st["completed"] == len(reqs)
        assert st["peak_bytes_in_flight"] <= budget
        for t in tickets:
            s.wait(t)
    big = W.serve_request(np.random.default_rng(1), 3000, False, 0.0, False)
    with E.Server(slots=1, hbm_budget=1000) as tiny:
        with pytest.raises(E.WbfmmError) as ei:
            tiny.submit(big, E.FP64)
        assert ei.value.code == -6


@pytest.mark.gpu
def test_failed_request_is_isolated(gpu_lib):
    reqs = list(W.serving_stream(6, seed=25, n_hi=2e4))
    bad = W.serve_request(np.random.default_rng(3), 2000, False, 0.0, False)
    bad.xs = bad.xs.copy()
    bad.xs[17] = bad.x0 - 1.0        # outside the tree cube
    with E.Server(slots=4) as s:
        tb = s.submit(bad, E.FP32)
        tickets = [s.submit(p, _precision(p)) for p in reqs]
        with pytest.raises(E.WbfmmError) as ei:
            s.wait(tb)
        assert ei.value.code == -2
        for t in tickets:
            pot, grad = s.wait(t)
            assert np.all(np.isfinite(pot)) and np.all(np.isfinite(grad))


@pytest.mark.gpu
def test_largest_first_order(gpu_lib):
    """With the largest-first order, a free slot takes the arrived request of
    the largest footprint: on one slot, the requests queued behind the first
    start in decreasing size, and every field is the one the arrival order
    gives."""
    rng = np.random.default_rng(31)
    sizes = [3000, 9000, 5000, 20000, 12000, 7000]
    reqs = [W.serve_request(rng, n, False, 0.0, False) for n in sizes]
    for p in reqs:        # one tree shape, so that the footprint follows n
        p.depth = 3
        p.order_s = p.order_r = [0, 10, 10, 10]
    out = {}
    for lf in (False, True):
        with E.Server(slots=1, largest_first=lf) as s:
            tickets = [s.submit(p, E.FP64) for p in reqs]
            s.drain()
            starts = [s.times(t)[1] for t in tickets]
            out[lf] = [[a.copy() for a in s.wait(t)] for t in tickets]
        if lf:
            queued = sorted(range(len(reqs)), key=lambda i: starts[i])[1:]
            assert queued == sorted(queued, key=lambda i: -sizes[i]), (queued, starts)
    for a, b in zip(out[False], out[True]):
        for x, y in zip(a, b):
            assert rel(y, x) <= 1e-12
