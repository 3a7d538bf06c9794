"""Seeded synthetic point sets for the FMM workloads this library is measured on.

Each generator returns a :class:`Problem` holding FP64 host arrays in the
reference's layouts (points ``[n,3]``; Laplace strengths real ``[n]``;
Helmholtz strengths complex interleaved ``[2n]``).  The tree cube follows the
reference drivers' fit rule: origin = min - 0.01, width = max extent + 0.02
(tools/wbfmm-tree-calc.c.in:261-267), which keeps every point strictly inside
the cube as ``wbfmm_tree_add_points`` requires (src/boxes.c:148-153).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

LAPLACE = 1
HELMHOLTZ = 2


@dataclass
class Problem:
    name: str
    problem: int              # 1 Laplace, 2 Helmholtz
    depth: int
    order_s: list             # per level 0..depth
    order_r: list
    k: float
    xs: np.ndarray            # [ns,3]
    q: np.ndarray | None      # Laplace [ns]; Helmholtz [2ns]
    xt: np.ndarray            # [nt,3]
    normals: np.ndarray | None = None
    dipoles: np.ndarray | None = None
    x0: np.ndarray = field(default_factory=lambda: np.zeros(3))
    D: float = 1.0
    targets_are_sources: bool = False

    @property
    def ns(self) -> int:
        return self.xs.shape[0]

    @property
    def nt(self) -> int:
        return self.xt.shape[0]

    @property
    def points(self) -> int:
        """Points counted by the throughput metric: sources + distinct targets."""
        return self.ns + (0 if self.targets_are_sources else self.nt)


def fit_box(*point_sets, margin: float = 1e-2):
    """Origin and width as in the reference drivers' -b option."""
    lo = np.min([p.min(axis=0) for p in point_sets], axis=0)
    hi = np.max([p.max(axis=0) for p in point_sets], axis=0)
    D = float(np.max(hi - lo))
    return lo - margin, D + 2.0 * margin


def helmholtz_order(k: float, width: float, c: float = 1.8, lo: int = 6,
                    hi: int | None = 30) -> int:
    """p = ceil(kD + c*6^(2/3)*(kD)^(1/3)), clamped (kD = k * box width)."""
    kd = k * width
    p = math.ceil(kd + c * 6.0 ** (2.0 / 3.0) * kd ** (1.0 / 3.0))
    p = max(lo, p)
    if hi is not None:
        p = min(hi, p)
    return p


def _finish(p: Problem) -> Problem:
    pts = [p.xs] if p.targets_are_sources else [p.xs, p.xt]
    p.x0, p.D = fit_box(*pts)
    return p


def laplace_cube(n_src: int = 20000, n_tgt: int = 20000, depth: int = 4,
                 order: int = 12, seed: int = 1) -> Problem:
    """Laplace, uniform sources and separate uniform targets in [-0.5,0.5]^3."""
    rng = np.random.default_rng(seed)
    xs = rng.uniform(-0.5, 0.5, size=(n_src, 3))
    q = rng.standard_normal(n_src)
    xt = rng.uniform(-0.5, 0.5, size=(n_tgt, 3))
    orders = [0] + [order] * depth
    return _finish(Problem("laplace_cube", LAPLACE, depth, orders, list(orders),
                           0.0, xs, q, xt))


def helmholtz_cube(n: int = 1_000_000, k: float = 8.0, depth: int = 6,
                   seed: int = 2, lo: int = 6, hi: int = 30) -> Problem:
    """Helmholtz monopoles, uniform in the cube, targets = sources,
    complex N(0,1) strengths, per-level order from the box width."""
    rng = np.random.default_rng(seed)
    xs = rng.uniform(-0.5, 0.5, size=(n, 3))
    q = rng.standard_normal(2 * n)
    p = Problem("helmholtz_cube", HELMHOLTZ, depth, [0] * (depth + 1),
                [0] * (depth + 1), k, xs, q, xs, targets_are_sources=True)
    p = _finish(p)
    for lv in range(1, depth + 1):
        o = helmholtz_order(k, p.D / 2 ** lv, lo=lo, hi=hi)
        p.order_s[lv] = p.order_r[lv] = o
    return p


def helmholtz_sphere(n_src: int = 2_000_000, n_tgt: int = 500_000,
                     k: float = 40.0, depth: int = 7, seed: int = 3,
                     hi: int | None = None, lo: int = 6) -> Problem:
    """Helmholtz surface distribution: sources on a sphere r=0.45, first
    half monopoles and second half dipoles along the radial normal; targets
    on a concentric sphere r=0.49."""
    rng = np.random.default_rng(seed)

    def sphere(m, r):
        v = rng.standard_normal((m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        return v * r, v

    xs, nrm = sphere(n_src, 0.45)
    qc = rng.standard_normal(2 * n_src)
    dc = rng.standard_normal(2 * n_src)
    half = n_src // 2
    q = qc.copy(); q[2 * half:] = 0.0
    d = dc.copy(); d[: 2 * half] = 0.0
    xt, _ = sphere(n_tgt, 0.49)
    p = Problem("helmholtz_sphere", HELMHOLTZ, depth, [0] * (depth + 1),
                [0] * (depth + 1), k, xs, q, xt, normals=nrm, dipoles=d)
    p = _finish(p)
    for lv in range(1, depth + 1):
        o = helmholtz_order(k, p.D / 2 ** lv, lo=lo, hi=hi)
        p.order_s[lv] = p.order_r[lv] = o
    return p


def laplace_clusters(n: int = 16_000_000, depth: int = 8, order: int = 10,
                     seed: int = 5, nclusters: int = 8,
                     sigma: float = 0.05) -> Problem:
    """Laplace, points from isotropic Gaussian clusters clipped to the cube,
    targets = sources."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.4, 0.4, size=(nclusters, 3))
    which = rng.integers(0, nclusters, size=n)
    xs = centres[which] + sigma * rng.standard_normal((n, 3))
    np.clip(xs, -0.5, 0.5, out=xs)
    q = rng.standard_normal(n)
    orders = [0] + [order] * depth
    return _finish(Problem("laplace_clusters", LAPLACE, depth, orders,
                           list(orders), 0.0, xs, q, xs,
                           targets_are_sources=True))


def subsample(rng_seed: int, n_total: int, m: int) -> np.ndarray:
    rng = np.random.default_rng(rng_seed)
    return np.sort(rng.choice(n_total, size=min(m, n_total), replace=False))


# ----------------------------------------------------------- serving stream
# Orders for a 1e-6 relative-L2 field error, from the FP64-vs-direct-sum
# calibration of this engine (uniform cube and sphere surface, 1e5 points,
# mean leaf occupancy ~64): Laplace p = 14 gives 6e-8 (potential) and 5e-7
# (gradient); Helmholtz p_l = max(14, kw + 1.8*6^(2/3)*(kw)^(1/3)) gives at
# most 1.2e-7 and 5e-7 for k in [1, 30].
SERVE_LAPLACE_ORDER = 14
SERVE_HELMHOLTZ_FLOOR = 14


def serve_depth(n: int) -> int:
    """Depth for a mean leaf occupancy of about 64 points (at least 2)."""
    return int(min(8, max(2, round(math.log(max(n, 1) / 64.0, 8)))))


def serve_request(rng: np.random.Generator, n: int, helmholtz: bool, k: float,
                  sphere: bool, name: str = "request") -> Problem:
    """One request of the serving stream: targets = sources."""
    if sphere:
        v = rng.standard_normal((n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        xs = 0.45 * v
    else:
        xs = rng.uniform(-0.5, 0.5, size=(n, 3))
    problem = HELMHOLTZ if helmholtz else LAPLACE
    q = rng.standard_normal(2 * n if helmholtz else n)
    depth = serve_depth(n)
    p = Problem(name, problem, depth, [0] * (depth + 1), [0] * (depth + 1),
                k if helmholtz else 0.0, xs, q, xs, targets_are_sources=True)
    p = _finish(p)
    for lv in range(1, depth + 1):
        if helmholtz:
            o = helmholtz_order(k, p.D / 2 ** lv, lo=SERVE_HELMHOLTZ_FLOOR, hi=60)
        else:
            o = SERVE_LAPLACE_ORDER
        p.order_s[lv] = p.order_r[lv] = o
    return p


def serving_stream(n_requests: int = 4096, seed: int = 4, n_lo: float = 1e3,
                   n_hi: float = 3e5):
    """Yield the requests of the mixed serving stream: N log-uniform in
    [n_lo, n_hi], half Laplace and half Helmholtz with k ~ U[1, 30], sources
    in the cube or on the r = 0.45 sphere (fair coin), N(0,1) strengths
    (complex for Helmholtz), targets = sources."""
    rng = np.random.default_rng(seed)
    lo, hi = math.log(n_lo), math.log(n_hi)
    for i in range(n_requests):
        n = int(round(math.exp(rng.uniform(lo, hi))))
        helm = bool(rng.random() < 0.5)
        k = float(rng.uniform(1.0, 30.0)) if helm else 0.0
        sphere = bool(rng.random() < 0.5)
        yield serve_request(rng, n, helm, k, sphere, name=f"request{i}")


def poisson_arrivals(n: int, rate: float, seed: int = 104) -> np.ndarray:
    """Arrival times (s) of a Poisson process of `rate` requests per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
