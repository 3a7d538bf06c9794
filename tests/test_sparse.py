"""Sparse level storage (``SolverConfig.sparse``): a level's coefficient
arrays hold only the groups of eight sibling boxes whose parent holds
sources or targets (the reference always stores all 8^l boxes,
src/boxes.c:518-583).

* the fields equal the dense solve's with the same M2L kernels (the tile
  kernel, or the automatic choice of the lane kernel at low orders) and
  skip_empty, which sparse storage implies: FP64 and FP32,
  Laplace and Helmholtz (dipoles, the scaled FP32 Helmholtz M2L), targets
  equal to the sources and targets in boxes that hold no sources;
* the coefficients of levels 2..depth, expanded to Layout L, equal the
  dense arrays in the stored groups and are zero elsewhere;
* the stored groups of each level are the boxes of the level above that
  hold sources (the tree's box counts) or targets (the floor rule of
  src/boxes.c:585-634, counted on the host); the bytes follow from them;
* the calls that need dense Layout L arrays refuse a sparse solver;
* against the reference's own outputs (the golden fixtures) at 1e-10, and
  under graph replay bit for bit.
"""
import numpy as np
import pytest

from wbfmm_b200 import engine, workloads as W

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def separate_targets(seed=61):
    """Laplace sources in two clusters, targets in a third cluster that holds
    no sources (and some targets among the sources)."""
    rng = np.random.default_rng(seed)
    c = np.array([[-0.3, -0.3, -0.3], [0.25, -0.2, 0.3], [0.2, 0.3, -0.25]])
    xs = np.concatenate([c[0] + 0.04 * rng.standard_normal((20_000, 3)),
                         c[1] + 0.04 * rng.standard_normal((20_000, 3))])
    xt = np.concatenate([c[2] + 0.04 * rng.standard_normal((6_000, 3)),
                         c[0] + 0.04 * rng.standard_normal((2_000, 3))])
    q = rng.standard_normal(xs.shape[0])
    orders = [0] + [9] * 6
    return W._finish(W.Problem("laplace_separate", W.LAPLACE, 6, orders, list(orders), 0.0,
                               xs, q, xt))


def case_problem(case):
    if case == "laplace_clusters":
        return W.laplace_clusters(60_000, depth=6, order=8, seed=48)
    if case == "helmholtz_sphere":
        return W.helmholtz_sphere(40_000, 10_000, k=12.0, depth=5, seed=47, hi=12)
    if case == "helmholtz_low_kw":
        # order 14 with 2 k w in [0.8, 1] at the leaf level: the FP32 form's
        # scaled Helmholtz M2L
        return W.serve_request(np.random.default_rng(91), 150_000, True, 7.0, True)
    if case == "separate_targets":
        return separate_targets()
    raise ValueError(case)


def solve(p, precision, sparse, keep=False, mode=3):
    cfg = engine.SolverConfig.from_problem(p, precision, skip_empty=True, sparse=sparse)
    s = engine.Solver(cfg)
    s.set_m2l_kernel(mode)       # 3: the tile kernel; 1: lanes at low orders, tiles above
    s.set_sources(p.xs, p.normals).set_strengths(p.q, p.dipoles).set_targets(p.xt).run()
    out = s.field()
    if keep:
        return s, out
    s.close()
    return out


@pytest.mark.parametrize("mode", [1, 3])
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
@pytest.mark.parametrize("case", ["laplace_clusters", "helmholtz_sphere", "helmholtz_low_kw",
                                  "separate_targets"])
def test_sparse_fields_match_dense(gpu_lib, case, precision, mode):
    p = case_problem(case)
    dense = solve(p, precision, False, mode=mode)
    sparse = solve(p, precision, True, mode=mode)
    # the same kernels in the same order on the same values: equal up to
    # rounding (in practice bit for bit)
    tol = 1e-13 if precision == engine.FP64 else 1e-6
    for a, b in zip(sparse, dense):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, b) < tol, (case, rel_l2(a, b))


def host_stored_groups(s, p, level):
    """Boxes of level - 1 that hold sources (the tree's counts) or targets
    (leaf boxes by the floor rule, then their ancestors)."""
    _, _, bn = s.tree(level - 1)
    occ = bn > 0
    nl = 2 ** p.depth
    ijk = np.floor((p.xt - p.x0) / (p.D / nl)).astype(np.int64)
    ijk = np.clip(ijk, 0, nl - 1) >> (p.depth - (level - 1))
    occ[morton(ijk)] = True
    return occ


def morton(ijk):
    out = np.zeros(ijk.shape[0], dtype=np.int64)
    for bit in range(21):
        for a in range(3):
            out |= ((ijk[:, a] >> bit) & 1) << (3 * bit + a)
    return out


@pytest.mark.parametrize("case", ["laplace_clusters", "separate_targets", "helmholtz_sphere"])
def test_sparse_coefficients_and_storage(gpu_lib, case):
    p = case_problem(case)
    sd, _ = solve(p, engine.FP64, False, keep=True)
    ss, _ = solve(p, engine.FP64, True, keep=True)
    w = 2 if p.problem == W.HELMHOLTZ else 1
    total_groups = total_bytes = 0
    try:
        for lv in range(1, p.depth + 1):
            occ = host_stored_groups(ss, p, lv)
            g, b = ss.coefficient_storage(lv)
            assert g == int(occ.sum()), (lv, g, int(occ.sum()))
            ncs = (p.order_s[lv] + 1) ** 2
            ncr = (p.order_r[lv] + 1) ** 2
            assert b == g * 8 * (ncs + ncr) * w * 8
            gd, bd = sd.coefficient_storage(lv)
            assert gd == 8 ** (lv - 1) and bd == gd * 8 * (ncs + ncr) * w * 8
            total_groups += g
            total_bytes += b
            if lv < 2:
                continue    # the passes write levels 2..depth (src/pass.c)
            for arr_s, arr_d, nc in zip(ss.coefficients(lv), sd.coefficients(lv), (ncs, ncr)):
                gs = arr_s.reshape(8 ** (lv - 1), 8 * nc * w)
                gdn = arr_d.reshape(8 ** (lv - 1), 8 * nc * w)
                assert np.all(gs[~occ] == 0.0)
                if np.any(gdn[occ]):
                    assert rel_l2(gs[occ], gdn[occ]) < 1e-13, lv
                else:
                    assert not np.any(gs[occ])
        assert ss.coefficient_storage(0) == (total_groups, total_bytes)
        assert total_bytes < sd.coefficient_storage(0)[1]
    finally:
        ss.close()
        sd.close()


def test_sparse_refuses_dense_only_calls(gpu_lib):
    p = W.laplace_clusters(20_000, depth=5, order=6, seed=63)
    cfg = engine.SolverConfig.from_problem(p, engine.FP64, sparse=True)
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
        with pytest.raises(engine.WbfmmError, match="dense"):
            s.hessian()
        with pytest.raises(engine.WbfmmError, match="dense"):
            s.target_bases()
        import ctypes as C
        a, b = C.c_void_p(), C.c_void_p()
        rc = s.lib.wbfmm_b200_coefficient_pointers(s.h, 3, C.byref(a), C.byref(b))
        assert rc != 0
    bad = engine.SolverConfig.from_problem(p, engine.FP64, sparse=True)
    bad.managed = True
    with pytest.raises(engine.WbfmmError, match="managed"):
        engine.Solver(bad)


def test_sparse_repeated_geometry(gpu_lib):
    """New targets after a solve rebuild the group maps; the fields follow."""
    p = separate_targets(64)
    cfg = engine.SolverConfig.from_problem(p, engine.FP64, skip_empty=True, sparse=True)
    q2 = np.random.default_rng(65).standard_normal(p.ns)
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
        g1 = s.coefficient_storage(0)[0]
        s.set_targets(p.xs[:5000]).run()
        a = s.field()
        g2 = s.coefficient_storage(0)[0]
        s.set_strengths(q2).run()
        c = s.field()
    assert g2 != g1
    p2 = W.Problem(p.name, p.problem, p.depth, p.order_s, p.order_r, 0.0, p.xs, p.q,
                   p.xs[:5000].copy())
    p2.x0, p2.D = p.x0, p.D
    ref = solve(p2, engine.FP64, False)
    for x, y in zip(a, ref):
        assert rel_l2(x, y) < 1e-13
    p2.q = q2
    ref2 = solve(p2, engine.FP64, False)
    for x, y in zip(c, ref2):
        assert rel_l2(x, y) < 1e-13


def test_sparse_deep_clusters(gpu_lib):
    """A deep tree of clustered points (2e6 points, depth 8, the lane M2L at
    order 6): sparse and dense storage give the same fields, and the sparse
    arrays are a fraction of the dense ones."""
    p = W.laplace_clusters(2_000_000, depth=8, order=6, seed=66)
    dense = solve(p, engine.FP32, False, mode=1)
    ss, sparse = solve(p, engine.FP32, True, keep=True, mode=1)
    try:
        g, b = ss.coefficient_storage(0)
        dense_bytes = sum(8 ** lv * 2 * (p.order_s[lv] + 1) ** 2 * 4 for lv in range(1, p.depth + 1))
        assert b < dense_bytes / 4, (b, dense_bytes)
    finally:
        ss.close()
    for a, c in zip(sparse, dense):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, c) < 1e-6, rel_l2(a, c)


def test_sparse_graph_replay(gpu_lib):
    """Repeated solves with new strengths through the captured graph (the
    group maps are built by the first, uncaptured run): the same fields as
    direct runs, bit for bit."""
    p = separate_targets(67)
    rng = np.random.default_rng(68)
    qs = [rng.standard_normal(p.ns) for _ in range(3)]
    cfg = engine.SolverConfig.from_problem(p, engine.FP32, sparse=True)
    refs = []
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs).set_targets(p.xt)
        for q in qs:
            s.set_strengths(q).run()
            refs.append(s.field())
    with engine.Solver(cfg) as s:
        s.set_deferred_checks(True)
        s.set_sources(p.xs).set_targets(p.xt)
        for q, ref in zip(qs, refs):
            s.set_strengths(q).run_graph()
            s.wait()
            for a, b in zip(s.field(), ref):
                assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["laplace_small", "helmholtz_small", "laplace_dipole_small",
                                  "helmholtz_dipole_small"])
def test_sparse_matches_reference_golden(gpu_lib, name):
    """Sparse storage against the reference's own outputs (the golden
    fixtures: the unmodified reference FMM at the same depth and orders,
    monopoles and dipoles), 1e-10 as the dense plain form."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    p = W.Problem(name, int(z["problem"]), int(z["depth"]), list(z["order_s"]),
                  list(z["order_r"]), float(z["k"]), z["xs"], z["q"] if z["q"].size else None,
                  z["xt"], normals=z["normals"] if z["normals"].size else None,
                  dipoles=z["dipoles"] if z["dipoles"].size else None)
    p.x0, p.D = z["x0"], float(z["D"])
    has_grad = z["grad"].size > 0
    field = engine.POTENTIAL | (engine.GRADIENT if has_grad else 0)
    cfg = engine.SolverConfig.from_problem(p, engine.FP64, field, sparse=True)
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs, p.normals).set_strengths(p.q, p.dipoles).set_targets(p.xt).run()
        pot, grad = s.field()
    assert rel_l2(pot, z["pot"]) < 1e-10
    if has_grad:
        assert rel_l2(grad, z["grad"]) < 1e-10
