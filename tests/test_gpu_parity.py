"""Parity of the GPU engine with the reference, through the C ABI.

* plain FP64 form: field and gradient within 1e-10 (relative L2 and relative
  max) of the reference CPU FMM at the same depth and orders, against the
  committed golden fixtures and, where the reference library is built, live;
* tree: `t->ip` and every box {i, n} bit-exact, including the values the
  reference's refinement leaves in non-leaf levels;
* coefficients: every level's singular and regular expansions, Layout L,
  within 1e-10 of the reference;
* FP32 form: within 1e-6 relative L2 of the plain FP64 form.
"""
import glob
import os

import numpy as np
import pytest

from oracle.oracle_api import HELMHOLTZ, LAPLACE, level_box_offsets
from wbfmm_b200 import engine, workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_FP64 = 1e-10
TOL_FP32 = 1e-6


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def load_case(path):
    z = np.load(path)
    p = W.Problem(os.path.basename(path)[:-4], int(z["problem"]), int(z["depth"]),
                  list(z["order_s"]), list(z["order_r"]), float(z["k"]), z["xs"],
                  z["q"] if z["q"].size else None, z["xt"],
                  normals=z["normals"] if z["normals"].size else None,
                  dipoles=z["dipoles"] if z["dipoles"].size else None)
    p.x0, p.D = z["x0"], float(z["D"])
    return p, z


def run(p, precision=engine.FP64, field=engine.POTENTIAL | engine.GRADIENT,
        keep=False):
    cfg = engine.SolverConfig.from_problem(p, precision, field)
    s = engine.Solver(cfg)
    s.set_sources(p.xs, p.normals)
    s.set_strengths(p.q, p.dipoles)
    s.set_targets(p.xt)
    s.run()
    pot, grad = s.field()
    if keep:
        return s, pot, grad
    s.close()
    return pot, grad


@pytest.mark.parametrize("path", sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                                        if not os.path.basename(p).startswith(("dropin_", "direct_"))),
                         ids=lambda x: os.path.basename(x)[:-4])
def test_golden_fp64(gpu_lib, path):
    p, z = load_case(path)
    has_grad = z["grad"].size > 0
    field = engine.POTENTIAL | (engine.GRADIENT if has_grad else 0)
    s, pot, grad = run(p, field=field, keep=True)
    try:
        assert rel_l2(pot, z["pot"]) < TOL_FP64
        assert rel_max(pot, z["pot"]) < TOL_FP64
        if has_grad:
            assert rel_l2(grad, z["grad"]) < TOL_FP64
            assert rel_max(grad, z["grad"]) < TOL_FP64
        # tree: bit-exact permutation and box ranges at every level
        offs = level_box_offsets(p.depth)
        for lv in range(p.depth + 1):
            ip, bi, bn = s.tree(lv)
            ref = z["boxes"][offs[lv]:offs[lv + 1]]
            assert np.array_equal(ip, z["ip"])
            assert np.array_equal(bi, ref[:, 0]), f"box .i differs at level {lv}"
            assert np.array_equal(bn, ref[:, 1]), f"box .n differs at level {lv}"
    finally:
        s.close()


@pytest.mark.parametrize("name", ["laplace", "helmholtz"])
def test_coefficients_every_level(gpu_lib, reference, name):
    if name == "laplace":
        p = W.laplace_cube(3000, 800, depth=4, order=7, seed=21)
    else:
        p = W.helmholtz_cube(3000, k=6.0, depth=4, seed=22)
        p.xt = p.xt[:800]
    r = reference.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs,
                      p.q, p.xt, k=p.k, want_coeffs=True)
    s, pot, grad = run(p, keep=True)
    try:
        w = 2 if p.problem == HELMHOLTZ else 1
        os_ = ors = 0
        for lv in range(1, p.depth + 1):
            ns = 8 ** lv * (p.order_s[lv] + 1) ** 2 * w
            nr = 8 ** lv * (p.order_r[lv] + 1) ** 2 * w
            ms, mr = s.coefficients(lv)
            if lv >= 2:
                assert rel_max(ms, r["mps"][os_:os_ + ns]) < TOL_FP64, f"mps level {lv}"
                assert rel_max(mr, r["mpr"][ors:ors + nr]) < TOL_FP64, f"mpr level {lv}"
            os_ += ns
            ors += nr
        assert rel_l2(pot, r["pot"]) < TOL_FP64
        assert rel_l2(grad, r["grad"]) < TOL_FP64
    finally:
        s.close()


def test_laplace_c1_reference_config(gpu_lib, reference):
    """Laplace, 2e4 sources / 2e4 targets, depth 4, order 12: the
    reference's own CPU-runnable configuration."""
    p = W.laplace_cube(20000, 20000, depth=4, order=12, seed=1)
    r = reference.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs,
                      p.q, p.xt, nthreads=os.cpu_count() or 1)
    pot, grad = run(p)
    assert rel_l2(pot, r["pot"]) < TOL_FP64
    assert rel_l2(grad, r["grad"]) < TOL_FP64
    assert rel_max(pot, r["pot"]) < TOL_FP64


def test_helmholtz_per_level_orders(gpu_lib, reference):
    """Helmholtz with per-level orders from the box width (orders differ
    between levels, exercising M2M/L2L between different orders)."""
    p = W.helmholtz_cube(30000, k=8.0, depth=5, seed=2)
    assert len(set(p.order_s[2:])) > 1
    p.xt = p.xs[:3000]
    r = reference.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs,
                      p.q, p.xt, k=p.k, nthreads=os.cpu_count() or 1)
    pot, grad = run(p)
    assert rel_l2(pot, r["pot"]) < TOL_FP64
    assert rel_l2(grad, r["grad"]) < TOL_FP64


@pytest.mark.parametrize("name", ["laplace_small", "helmholtz_small"])
def test_fp32_form_vs_fp64(gpu_lib, name):
    p, z = load_case(os.path.join(GOLDEN, name + ".npz"))
    pot64, grad64 = run(p, engine.FP64)
    pot32, grad32 = run(p, engine.FP32)
    assert rel_l2(pot32, pot64) < TOL_FP32
    assert rel_l2(grad32, grad64) < TOL_FP32


def test_direct_sum_accuracy(gpu_lib):
    """FMM error against the FP64 direct sum is the truncation error of the
    expansion order (checked loosely; parity is checked above)."""
    p, z = load_case(os.path.join(GOLDEN, "laplace_small.npz"))
    pot, grad = run(p)
    assert rel_l2(pot, z["direct_pot"]) < 1e-4
    assert rel_l2(grad, z["direct_grad"]) < 1e-3


def test_domain_error(gpu_lib):
    p = W.laplace_cube(500, 100, depth=2, order=4, seed=3)
    cfg = engine.SolverConfig.from_problem(p)
    with engine.Solver(cfg) as s:
        xs = p.xs.copy()
        xs[7] = p.x0  # on the cube's corner: not strictly inside
        with pytest.raises(engine.WbfmmError) as e:
            s.set_sources(xs)
        assert e.value.code == -2


def test_deferred_checks(gpu_lib):
    """With deferred checks the set calls do not wait: a source or target
    outside the cube is reported by run / wait, and a valid solve queued with
    run_async gives the fields of run."""
    p = W.laplace_cube(3000, 500, depth=3, order=6, seed=3)
    cfg = engine.SolverConfig.from_problem(p)
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
        ref = s.field()
    with engine.Solver(cfg) as s:
        s.set_deferred_checks(True)
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run_async().wait()
        for a, b in zip(s.field(), ref):
            assert np.array_equal(a, b)
        xs = p.xs.copy()
        xs[7] = p.x0
        s.set_sources(xs).set_strengths(p.q).set_targets(p.xt)   # no error yet
        with pytest.raises(engine.WbfmmError) as e:
            s.run()
        assert e.value.code == -2
        xt = p.xt.copy()
        xt[3] = p.x0 + 2.0 * p.D
        s.set_sources(p.xs).set_strengths(p.q).set_targets(xt).run_async()
        with pytest.raises(engine.WbfmmError) as e:
            s.wait()
        assert e.value.code == -2
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()   # recovers
        for a, b in zip(s.field(), ref):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("name,precision", [("laplace", engine.FP64), ("helmholtz", engine.FP64),
                                            ("laplace", engine.FP32), ("helmholtz", engine.FP32)])
def test_m2l_lane_kernel_matches_generic(gpu_lib, name, precision):
    """The lane-per-pair M2L and the generic warp M2L compute the same
    translations (orders 2..8 cover both kernels' ranges here)."""
    if name == "laplace":
        p = W.laplace_cube(20000, 3000, depth=5, order=7, seed=41)
    else:
        p = W.helmholtz_cube(20000, k=6.0, depth=5, seed=42)
        p.xt = p.xt[:3000]
    outs = []
    for lanes in (True, False):
        cfg = engine.SolverConfig.from_problem(p, precision)
        with engine.Solver(cfg) as s:
            s.set_m2l_kernel(lanes)
            s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
            outs.append(s.field())
    tol = 1e-12 if precision == engine.FP64 else 1e-5
    for a, b in zip(outs[0], outs[1]):
        assert rel_l2(a, b) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
@pytest.mark.parametrize("case", ["laplace13", "laplace16", "helmholtz_k6_floor11",
                                  "helmholtz_k20_floor9"])
def test_m2l_kernels_agree_at_high_order(gpu_lib, case, precision):
    """The offset-major tile M2L (mode 3), the lane-per-pair M2L where
    instantiated (mode 2) and the warp-per-target M2L (mode 0) compute the
    same translations at the orders of the served stream."""
    if case.startswith("laplace"):
        p = W.laplace_cube(30000, 3000, depth=4, order=int(case[7:]), seed=43)
    else:
        k = float(case.split("_")[1][1:])
        lo = int(case.split("floor")[1])
        p = W.helmholtz_cube(30000, k=k, depth=4, seed=44, lo=lo, hi=40)
        p.xt = p.xt[:3000]
        p.targets_are_sources = False
    outs = {}
    for mode in (0, 2, 3):
        cfg = engine.SolverConfig.from_problem(p, precision)
        with engine.Solver(cfg) as s:
            s.set_m2l_kernel(mode)
            s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
            outs[mode] = s.field()
    tol = 1e-12 if precision == engine.FP64 else 2e-5
    for mode in (2, 3):
        for a, b in zip(outs[mode], outs[0]):
            assert rel_l2(a, b) < tol, (mode, rel_l2(a, b))


@pytest.mark.gpu
@pytest.mark.parametrize("order", [8, 10, 12, 14, 15])
def test_laplace_m2l_tensor_cores(gpu_lib, order):
    """The Laplace FP32 M2L on the tensor cores (mode 4: dense shift
    operators, tcgen05 3xTF32 products accumulated in FP32) against the
    offset-major tile kernel (mode 3) and the FP64 form: every level of a
    depth-4 tree (split sums on the small levels, one pass on level 4)."""
    p = W.laplace_cube(30000, 3000, depth=4, order=order, seed=47)
    outs = {}
    for prec, mode in ((engine.FP64, 1), (engine.FP32, 3), (engine.FP32, 4)):
        cfg = engine.SolverConfig.from_problem(p, prec)
        with engine.Solver(cfg) as s:
            s.set_m2l_kernel(mode)
            s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
            outs[(prec, mode)] = s.field()
    tc, tiles, f64 = outs[(engine.FP32, 4)], outs[(engine.FP32, 3)], outs[(engine.FP64, 1)]
    for a, b, c in zip(tc, tiles, f64):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, c) < 2e-6, rel_l2(a, c)
        assert rel_l2(a, b) < 2e-6, rel_l2(a, b)


@pytest.mark.gpu
def test_laplace_m2l_tensor_cores_target_lists(gpu_lib):
    """The tensor-core M2L on the per-child-type target lists and source
    masks of skip_empty (clustered points, order 10, depth 6)."""
    p = W.laplace_clusters(60_000, depth=6, order=10, seed=48)
    outs = {}
    for skip, mode in ((False, 3), (True, 4)):
        cfg = engine.SolverConfig.from_problem(p, engine.FP32, skip_empty=skip)
        with engine.Solver(cfg) as s:
            s.set_m2l_kernel(mode)
            s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
            outs[mode] = s.field()
    for a, b in zip(outs[4], outs[3]):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, b) < 2e-6, rel_l2(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 2, 3])
def test_laplace_fp32_deep_levels(gpu_lib, mode):
    """Laplace FP32 at depth 7, order 10, on clustered points: S|R / t^(n+l+1)
    at the nearest list-4 distance (t = 2/128, n + l = 20) is beyond the
    FP32 range, so each M2L kernel must apply it in scaled form.  The FP32
    field is finite and agrees with the FP64 form and the direct sum."""
    p = W.laplace_clusters(200_000, depth=7, order=10, seed=45)
    cfg32 = engine.SolverConfig.from_problem(p, engine.FP32)
    assert engine.fp32_range_ok(cfg32)
    outs = {}
    for prec in (engine.FP64, engine.FP32):
        cfg = engine.SolverConfig.from_problem(p, prec)
        with engine.Solver(cfg) as s:
            s.set_m2l_kernel(mode)
            s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
            outs[prec] = s.field()
    for a in outs[engine.FP32]:
        assert np.all(np.isfinite(a))
    for a, b in zip(outs[engine.FP32], outs[engine.FP64]):
        assert rel_l2(a, b) < 1e-5, rel_l2(a, b)
    idx = W.subsample(46, p.nt, 2000)
    dpot, dgrad = engine.direct(p.problem, p.xs, p.q, p.xt[idx])
    pot, grad = outs[engine.FP32]
    assert rel_l2(pot[idx], dpot) < 1e-4
    assert rel_l2(grad.reshape(-1, 3)[idx].ravel(), dgrad) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cube_k7.8_n200000", "cube_k6.6_n190000", "sphere_k7_n150000"])
def test_helmholtz_fp32_scaled_m2l(gpu_lib, case):
    """Helmholtz at order 14 with k w just below the unscaled FP32 range of
    the leaf level's (S|R) table (2 k w in [0.8, 1]): those levels run the
    scaled M2L (sources x 2^(e l), table x 2^(-e (n + l)), results x
    2^(e n)); the range rule admits the FP32 form, whose fields are finite
    and within 1.5e-6 of the FP64 form and of the direct sum."""
    kind, kk, nn = case.split("_")
    k, n = float(kk[1:]), int(nn[1:])
    rng = np.random.default_rng(91)
    p = W.serve_request(rng, n, True, k, kind == "sphere")
    assert p.depth == 4
    assert 0.8 <= 2 * k * p.D / 16 < 1.02          # scaled at the leaf level
    skip = kind == "sphere"
    cfg32 = engine.SolverConfig.from_problem(p, engine.FP32, skip_empty=skip)
    assert engine.fp32_range_ok(cfg32)
    outs = {}
    for prec in (engine.FP64, engine.FP32):
        cfg = engine.SolverConfig.from_problem(p, prec, skip_empty=skip)
        with engine.Solver(cfg) as s:
            s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xs).run()
            outs[prec] = s.field()
    for a in outs[engine.FP32]:
        assert np.all(np.isfinite(a))
    for a, b in zip(outs[engine.FP32], outs[engine.FP64]):
        assert rel_l2(a, b) < 1.5e-6, rel_l2(a, b)
    idx = W.subsample(93, p.ns, 1500)
    dpot, dgrad = engine.direct(p.problem, p.xs, p.q, p.xs[idx], k=p.k)
    pot, grad = outs[engine.FP32]
    assert rel_l2(pot.reshape(-1, 2)[idx].ravel(), dpot) < 1.5e-6
    assert rel_l2(grad.reshape(-1, 6)[idx].ravel(), dgrad) < 1.5e-6


def test_helmholtz_fp32_rule_low_kw(gpu_lib):
    """Below 2 k w = 0.8 at the leaves the FP32 form loses accuracy to
    cancellation (low-frequency regime); the range rule sends such requests
    to the FP64 form."""
    p = W.serve_request(np.random.default_rng(92), 40_000, True, 1.5, False)
    assert 2 * 1.5 * p.D / 2 ** p.depth < 0.8
    assert not engine.fp32_range_ok(engine.SolverConfig.from_problem(p, engine.FP32))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
@pytest.mark.parametrize("mode", [0, 2, 3])
@pytest.mark.parametrize("case", ["helmholtz_spheres", "laplace_clusters"])
def test_skip_empty_matches_dense(gpu_lib, case, mode, precision):
    """Sparse geometries: with skip_empty the M2L kernels walk the per-level
    lists of boxes that hold targets instead of every box; the fields at the
    targets are those of the dense solve."""
    if case == "helmholtz_spheres":
        p = W.helmholtz_sphere(40_000, 10_000, k=12.0, depth=5, seed=47, hi=12)
    else:
        p = W.laplace_clusters(60_000, depth=6, order=8, seed=48)
    outs = {}
    for skip in (False, True):
        cfg = engine.SolverConfig.from_problem(p, precision, skip_empty=skip)
        with engine.Solver(cfg) as s:
            s.set_m2l_kernel(mode)
            s.set_sources(p.xs, p.normals).set_strengths(p.q, p.dipoles).set_targets(p.xt).run()
            outs[skip] = s.field()
    tol = 1e-13 if precision == engine.FP64 else 1e-6
    for a, b in zip(outs[True], outs[False]):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, b) < tol, rel_l2(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("xmax", [3.2, 100.0, 1e4])
def test_near_field_sincos(gpu_lib, xmax):
    """The FP32 P2P's own sine/cosine (Cody-Waite reduction, Taylor
    polynomials) is as accurate as CUDA's sincosf at the same arguments."""
    ours, cuda = engine.selftest_sincos(xmax, 200_000)
    assert ours <= max(1.5 * cuda, 2.0e-7), (ours, cuda)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
@pytest.mark.parametrize("case", ["laplace", "helmholtz"])
def test_graph_replay(gpu_lib, case, precision):
    """Repeated solves on one tree with new strengths: the captured graph of
    the passes gives exactly the fields of a direct run, and a change of the
    targets makes the next call capture again."""
    if case == "laplace":
        p = W.laplace_cube(20000, 3000, depth=4, order=8, seed=51)
    else:
        p = W.helmholtz_cube(20000, k=6.0, depth=4, seed=52)
        p.xt = p.xt[:3000]
        p.targets_are_sources = False
    rng = np.random.default_rng(53)
    qs = [rng.standard_normal(p.q.shape) for _ in range(3)]
    cfg = engine.SolverConfig.from_problem(p, precision)
    refs = []
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs).set_targets(p.xt)
        for q in qs:
            s.set_strengths(q).run()
            refs.append(s.field())
    with engine.Solver(cfg) as s:
        s.set_deferred_checks(True)
        s.set_sources(p.xs).set_targets(p.xt)
        s.set_strengths(qs[0]).run_graph().wait()          # runs and captures
        for q, ref in zip(qs, refs):
            n1 = s.kernel_launches()
            s.set_strengths(q).run_graph().wait()          # graph launches
            per_graph = s.kernel_launches() - n1
            for a, b in zip(s.field(), ref):
                assert np.array_equal(a, b)
        n2 = s.kernel_launches()
        s.set_strengths(qs[0]).run_async().wait()          # the same passes, launched directly
        assert per_graph == s.kernel_launches() - n2
        xt2 = p.xt[::2].copy()
        s.set_targets(xt2).set_strengths(qs[1]).run_graph().wait()   # captures again
        with engine.Solver(cfg) as s2:
            s2.set_sources(p.xs).set_strengths(qs[1]).set_targets(xt2).run()
            for a, b in zip(s.field(), s2.field()):
                assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
def test_leaf_order(gpu_lib, precision):
    """Sorting the sources by leaf box only gives the same boxes, the same
    points in every leaf (in input order there) and, up to the order of
    summation, the same fields."""
    p = W.helmholtz_cube(30000, k=6.0, depth=4, seed=54)
    outs, trees = [], []
    for lo in (False, True):
        cfg = engine.SolverConfig.from_problem(p, precision, leaf_order=lo)
        with engine.Solver(cfg) as s:
            s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
            outs.append(s.field())
            trees.append(s.tree(p.depth))
    (ip0, bi0, bn0), (ip1, bi1, bn1) = trees
    assert np.array_equal(bi0, bi1) and np.array_equal(bn0, bn1)
    for b in np.nonzero(bn0)[0][:2000]:
        a, c = ip0[bi0[b]:bi0[b] + bn0[b]], ip1[bi1[b]:bi1[b] + bn1[b]]
        assert np.array_equal(np.sort(a), c)          # input order inside the leaf
    tol = 1e-12 if precision == engine.FP64 else 2e-6
    for a, b in zip(outs[0], outs[1]):
        assert rel_l2(a, b) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 1000, 3_000_001])
def test_error_norms(gpu_lib, n):
    """The GPU accuracy reduction agrees with numpy (relative L2 and max)."""
    rng = np.random.default_rng(55)
    ref = rng.standard_normal(n)
    f = ref + 1e-7 * rng.standard_normal(n)
    l2, mx = engine.error_norms(f, ref)
    assert abs(l2 - np.linalg.norm(f - ref) / np.linalg.norm(ref)) <= 1e-12 * l2
    assert mx == np.max(np.abs(f - ref)) / np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
def test_laplace_curl(gpu_lib, precision):
    """The FMM curl of a vector potential (three source components) against
    the direct curl built from the oracle's direct gradients, whose
    convention the CPU suite pins to the reference's direct curl."""
    from oracle.oracle_api import Restatement, curl_from_gradients
    p = W.laplace_cube(20000, 2000, depth=4, order=12, seed=62)
    q3 = np.random.default_rng(63).standard_normal((p.ns, 3))
    with engine.Solver(engine.SolverConfig.from_problem(p, precision)) as s:
        s.set_sources(p.xs).set_targets(p.xt)
        curl = s.laplace_curl(q3)
    ora = Restatement()
    g = [ora.direct(LAPLACE, p.xs, q3[:, c].copy(), p.xt, pot=False, grad=True)[1]
         for c in range(3)]
    ref = curl_from_gradients(g)
    tol = 2e-6 if precision == engine.FP64 else 5e-6
    assert rel_l2(curl.ravel(), ref.ravel()) < tol, rel_l2(curl.ravel(), ref.ravel())


def _direct_hessian(xs, q, xt, chunk=256):
    """d_a d_b of sum q / (4 pi r) at xt (self terms r <= 1e-6 excluded)."""
    out = np.zeros((xt.shape[0], 3, 3))
    for i in range(0, xt.shape[0], chunk):
        d = xt[i:i + chunk, None, :] - xs[None, :, :]
        r2 = np.einsum("tsk,tsk->ts", d, d)
        ok = r2 > 1e-12
        r2 = np.where(ok, r2, 1.0)
        r = np.sqrt(r2)
        w3 = np.where(ok, q[None, :] / (4 * np.pi * r2 * r), 0.0)
        w5 = 3.0 * w3 / r2
        out[i:i + chunk] = (np.einsum("ts,tsa,tsb->tab", w5, d, d)
                            - np.einsum("ts->t", w3)[:, None, None] * np.eye(3))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
def test_laplace_hessian(gpu_lib, precision):
    """Second derivatives of the Laplace potential (derived local
    expansions through the gradient L2P, plus the near-field monopoles)
    against a direct sum; symmetric as computed."""
    p = W.laplace_cube(20000, 1500, depth=4, order=12, seed=64)
    with engine.Solver(engine.SolverConfig.from_problem(p, precision)) as s:
        s.set_sources(p.xs).set_strengths(p.q).set_targets(p.xt).run()
        h = s.hessian()
        hfar = s.hessian(neighbours=False)
    ref = _direct_hessian(p.xs, p.q, p.xt)
    tol = 2e-5 if precision == engine.FP64 else 5e-5
    assert rel_l2(h.ravel(), ref.ravel()) < tol, rel_l2(h.ravel(), ref.ravel())
    assert np.abs(h - h.transpose(0, 2, 1)).max() <= 1e-6 * np.abs(h).max()
    # the far field alone is harmonic: the trace of its Hessian vanishes
    tr = np.trace(hfar, axis1=1, axis2=2)
    assert np.abs(tr).max() <= 1e-6 * np.abs(hfar).max()


@pytest.mark.gpu
def test_laplace_curl_gradient(gpu_lib):
    """The curl of a vector potential and its gradient (three source
    components) against the reference's own direct curl gradient
    (WBFMM_FIELD_CURL | WBFMM_FIELD_GRADIENT)."""
    from oracle.oracle_api import Reference, have_reference
    if not have_reference():
        pytest.skip("reference library not built")
    p = W.laplace_cube(20000, 600, depth=4, order=12, seed=65)
    q3 = np.random.default_rng(66).standard_normal((p.ns, 3))
    with engine.Solver(engine.SolverConfig.from_problem(p, engine.FP64)) as s:
        s.set_sources(p.xs).set_targets(p.xt)
        cg = s.laplace_curl_gradient(q3)
        curl = s.laplace_curl(q3)
    ref = Reference().direct_curl_gradient(p.xs, q3, p.xt)
    assert np.allclose(cg[:, :3], curl, rtol=0, atol=1e-12 * np.abs(curl).max())
    assert rel_l2(cg[:, :3].ravel(), ref[:, :3].ravel()) < 2e-6
    assert rel_l2(cg[:, 3:].ravel(), ref[:, 3:].ravel()) < 2e-5, rel_l2(cg[:, 3:].ravel(), ref[:, 3:].ravel())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [engine.FP64, engine.FP32])
@pytest.mark.parametrize("case", ["laplace", "helmholtz", "helmholtz_dipoles"])
def test_target_bases(gpu_lib, case, precision):
    """Potential at fixed targets from the precomputed bases and near-field
    weights (the reference's target-list strategy) against the L2P + P2P
    evaluation, for the first strengths and for new ones after a repeated
    solve; the far field alone without the near-field weights."""
    if case == "laplace":
        p = W.laplace_cube(20000, 3000, depth=4, order=10, seed=91)
    elif case == "helmholtz":
        p = W.helmholtz_cube(20000, k=6.0, depth=4, seed=92)
    else:
        p = W.helmholtz_sphere(20000, 3000, k=10.0, depth=4, seed=93)
    rng = np.random.default_rng(94)
    tol = 1e-12 if precision == engine.FP64 else 1e-6
    with engine.Solver(engine.SolverConfig.from_problem(p, precision)) as s:
        s.set_sources(p.xs, normals=p.normals)
        s.set_strengths(p.q, dipoles=p.dipoles).set_targets(p.xt).run()
        ref = s.field()[0]
        s.target_bases().evaluate_bases()
        got = s.field()[0]
        assert rel_l2(got, ref) < tol, rel_l2(got, ref)
        q2 = rng.standard_normal(p.q.shape)
        s.set_strengths(q2, dipoles=p.dipoles).run()
        ref2 = s.field()[0]
        s.evaluate_bases()
        assert rel_l2(s.field()[0], ref2) < tol, rel_l2(s.field()[0], ref2)
        s.evaluate_bases(neighbours=False)
        far = s.field()[0]
    with engine.Solver(engine.SolverConfig.from_problem(p, precision)) as s:
        s.set_sources(p.xs, normals=p.normals)
        s.set_strengths(q2, dipoles=p.dipoles).set_targets(p.xt).run()
        s.set_evaluation(engine.POTENTIAL, neighbours=False)
        s.evaluate()
        s.synchronize()
        far_ref = s.field()[0]
    assert rel_l2(far, far_ref) < tol, rel_l2(far, far_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["laplace", "helmholtz_dipoles"])
def test_fp64_with_fp32_near_field(gpu_lib, case):
    """An FP64 solve with its near field in the FP32 form's kernel
    (near_fp32) against the FP64 solve and the direct sum."""
    if case == "laplace":
        p = W.laplace_cube(20000, 2000, depth=4, order=12, seed=95)
    else:
        p = W.helmholtz_sphere(20000, 2000, k=8.0, depth=4, seed=96)
    outs = {}
    for near in (False, True):
        cfg = engine.SolverConfig.from_problem(p, engine.FP64, near_fp32=near)
        with engine.Solver(cfg) as s:
            s.set_sources(p.xs, normals=p.normals)
            s.set_strengths(p.q, dipoles=p.dipoles).set_targets(p.xt).run()
            outs[near] = s.field()
    # FP32 pair terms (FP64 sums per run of 8): within 1e-6 of the FP64 near
    # field (measured: 2.4e-7 on the dipole gradients, the most cancelling)
    for a, b in zip(outs[True], outs[False]):
        assert rel_l2(a, b) < 1e-6, rel_l2(a, b)
    # against the direct sum: the FP64 solve's own truncation error, unchanged
    idx = W.subsample(97, p.nt, 500)
    dpot, dgrad = engine.direct(p.problem, p.xs, p.q, p.xt[idx], k=p.k, normals=p.normals,
                                dipoles=p.dipoles)
    w = 2 if p.problem == engine.HELMHOLTZ else 1
    err = [rel_l2(outs[near][0].reshape(p.nt, w)[idx].ravel(), dpot) for near in (False, True)]
    assert abs(err[1] - err[0]) < 1e-6, err


def _edge_problem(case):
    rng = np.random.default_rng(71)
    if case == "coincident":
        # exact duplicates among the sources; targets on sources (excluded by
        # the r > 1e-6 cutoff, src/wbfmm.h:36) and on duplicated sources
        p = W.laplace_cube(3000, 600, depth=3, order=8, seed=72)
        p.xs[100:200] = p.xs[0:100]
        p.xt[:60] = p.xs[:60]
        p.xt[60:90] = p.xs[130:160]
    elif case == "faces":
        # points within 1e-9 D of every face of the cube (strictly inside)
        p = W.helmholtz_cube(4000, k=5.0, depth=3, seed=73)
        p.xs = p.xs.copy()
        for a in range(3):
            p.xs[a * 200:(a * 200 + 100), a] = p.x0[a] + 1e-9 * p.D
            p.xs[a * 200 + 100:(a + 1) * 200, a] = p.x0[a] + p.D * (1 - 1e-9)
        p.xt = p.xs
    elif case == "one_source":
        p = W.laplace_cube(1, 40, depth=2, order=6, seed=74)
        p.x0, p.D = np.array([-0.5, -0.5, -0.5]) - 0.01, 1.02
    else:   # "sparse": 60 points in a depth-5 tree (most boxes empty)
        p = W.helmholtz_cube(60, k=3.0, depth=5, seed=75)
    return p


@pytest.mark.parametrize("case", ["coincident", "faces", "one_source", "sparse"])
def test_edge_cases_match_reference(gpu_lib, reference, case):
    """Coincident points, points at the cube's faces, a single source and a
    nearly empty tree: fields equal to the reference FMM's (FP64, 1e-10)."""
    p = _edge_problem(case)
    r = reference.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs,
                      p.q, p.xt, k=p.k, nthreads=os.cpu_count() or 1)
    pot, grad = run(p)
    assert np.all(np.isfinite(pot)) and np.all(np.isfinite(grad))
    assert rel_l2(pot, r["pot"]) < TOL_FP64
    assert rel_l2(grad, r["grad"]) < TOL_FP64
