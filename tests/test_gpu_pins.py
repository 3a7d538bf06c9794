"""Parity pins for the paths the accuracy figures rest on, through the C ABI.

* the GPU FP64 direct sum (wbfmm_b200_direct, the accuracy oracle of every
  benchmark figure) against the reference's own direct sums
  (tests/golden/direct_sums.npz, from src/direct.c / src/direct-laplace.c);
* the drop-in direct-sum calls (wbfmm_total_field[_grad],
  wbfmm_laplace_field[_grad]) against the same calls of the reference
  library, argument for argument, including multi-component sources and
  the reference's normalisation of mixed sources;
* gradients of dipole sources, which the reference does not compute
  (src/local.c:259, src/direct.c:223): the FMM gradient is the derivative of
  the FMM potential (itself pinned to the reference at 1e-10) by central
  differences, and the GPU direct gradient equals the restatement's, whose
  own gradient the CPU suite checks by differences of the reference's
  potential;
* the benchmark's Helmholtz configuration at full size (1e6 points, k = 8,
  depth 6) against the reference FMM, and the FP32 form beside it.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle.oracle_api import HELMHOLTZ, LAPLACE
from wbfmm_b200 import engine, workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_DIRECT = 1e-12
TOL_FP64 = 1e-10
DIRECT_CASES = ("helm_mono", "helm_mixed", "lap_mono", "lap_dipole", "lap_mixed")


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def rel_max(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / np.max(np.abs(b)))


def direct_case(name):
    z = np.load(os.path.join(GOLDEN, "direct_sums.npz"))

    def g(a):
        key = f"{name}_{a}"
        if key not in z.files:
            return None
        v = z[key]
        return v if v.size else None

    c = {a: g(a) for a in ("xs", "xt", "q", "normals", "dipoles", "pot", "grad")}
    c["problem"], c["k"] = int(z[f"{name}_problem"]), float(z[f"{name}_k"])
    return c


@pytest.mark.parametrize("name", DIRECT_CASES)
def test_engine_direct_matches_reference(gpu_lib, name):
    """wbfmm_b200_direct (FP64, compensated, self-excluding) against the
    reference's direct sums on targets apart from every source.  For Laplace
    monopoles plus dipoles the reference leaves the 1/(4 pi) off the dipole
    term (src/direct-laplace.c:261-263); the engine keeps it, as the FMM
    does, so there the reference's value is the monopole sum plus 4 pi times
    the dipole sum."""
    c = direct_case(name)
    kw = dict(k=c["k"], normals=c["normals"], dipoles=c["dipoles"])
    pot, grad = engine.direct(c["problem"], c["xs"], c["q"], c["xt"], **kw)
    if name == "lap_mixed":
        mono, _ = engine.direct(c["problem"], c["xs"], c["q"], c["xt"], grad=False)
        dip, _ = engine.direct(c["problem"], c["xs"], None, c["xt"], grad=False, **kw)
        pot = mono + 4.0 * np.pi * dip
    assert rel_l2(pot, c["pot"]) < TOL_DIRECT
    assert rel_max(pot, c["pot"]) < TOL_DIRECT
    if c["grad"] is not None:
        assert rel_l2(grad, c["grad"]) < TOL_DIRECT
        assert rel_max(grad, c["grad"]) < TOL_DIRECT


_dp = C.POINTER(C.c_double)


def _bind_direct(lib):
    """The four direct-sum entry points of wbfmm.h (src/wbfmm.h), same
    signatures in the reference library and the drop-in."""
    helm = [C.c_double, _dp, C.c_int, _dp, C.c_int, _dp, C.c_int, _dp, C.c_int, C.c_int,
            C.c_int, _dp, _dp, C.c_int]
    lap = [_dp, C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int, C.c_int, _dp,
           _dp, C.c_int]
    out = {}
    for name, args in (("wbfmm_total_field", helm), ("wbfmm_total_field_grad", helm),
                       ("wbfmm_laplace_field", lap), ("wbfmm_laplace_field_grad", lap)):
        f = getattr(lib, name)
        f.restype = C.c_int
        f.argtypes = args
        out[name] = f
    return out


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _call_direct(fns, problem, grad, k, xs, src, sstr, nrm, dip, dstr, nq, xt, field0, fstr):
    """One direct-sum call per target, onto a copy of field0 (the reference
    adds into what the caller stored)."""
    out = field0.copy()
    ns = xs.shape[0]
    for j in range(xt.shape[0]):
        xf = np.ascontiguousarray(xt[j])
        f = out[j]
        if problem == HELMHOLTZ:
            fn = fns["wbfmm_total_field_grad" if grad else "wbfmm_total_field"]
            rc = fn(k, _p(xs), 3, _p(src), sstr, _p(nrm), 3, _p(dip), dstr, nq, ns, _p(xf),
                    _p(f), fstr)
        else:
            fn = fns["wbfmm_laplace_field_grad" if grad else "wbfmm_laplace_field"]
            rc = fn(_p(xs), 3, _p(src), sstr, nq, _p(nrm), 3, _p(dip), dstr, ns, _p(xf),
                    _p(f), fstr)
        assert rc == 0
    return out


# (name, problem, grad, monopoles, dipoles, nq): only calls the reference
# completes (it stops on dipole gradients and on dipole-only Helmholtz)
DROPIN_DIRECT = [
    ("helm_pot", HELMHOLTZ, False, True, False, 1),
    ("helm_pot_nq2", HELMHOLTZ, False, True, False, 2),
    ("helm_grad", HELMHOLTZ, True, True, False, 1),
    ("helm_grad_nq2", HELMHOLTZ, True, True, False, 2),
    ("helm_mixed_pot", HELMHOLTZ, False, True, True, 1),
    ("lap_pot", LAPLACE, False, True, False, 1),
    ("lap_pot_nq3", LAPLACE, False, True, False, 3),
    ("lap_grad", LAPLACE, True, True, False, 1),
    ("lap_grad_nq2", LAPLACE, True, True, False, 2),
    ("lap_dipole_pot", LAPLACE, False, False, True, 1),
    ("lap_mixed_pot", LAPLACE, False, True, True, 1),
]


@pytest.mark.parametrize("case", DROPIN_DIRECT, ids=[c[0] for c in DROPIN_DIRECT])
def test_dropin_direct_calls_match_reference(gpu_lib, reference, case):
    """The same wbfmm.h direct-sum call, argument for argument, on the
    drop-in and on the reference library: multi-component strengths with
    strides, field strides, and a field array that already holds values
    (the reference adds into it, and for Helmholtz mixed sources divides
    the first 2 nq entries by 4 pi afterwards)."""
    name, problem, grad, mono, dipole, nq = case
    rng = np.random.default_rng(301 + DROPIN_DIRECT.index(case))
    ns, nt = 700, 40
    xs = rng.uniform(-0.5, 0.5, (ns, 3))
    xt = rng.uniform(-0.5, 0.5, (nt, 3))
    w = 2 if problem == HELMHOLTZ else 1
    sstr = w * nq + 1                     # padded stride
    src = rng.standard_normal((ns, sstr)) if mono else None
    nrm = dip = None
    dstr = w * nq
    if dipole:
        nrm = rng.standard_normal((ns, 3))
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        dip = rng.standard_normal((ns, dstr))
    ncomp = (3 * w if grad else w)
    fstr = ncomp + 1 if nq > 1 else ncomp
    field0 = rng.standard_normal((nt, fstr * nq))
    kk = 5.7
    got = _call_direct(_bind_direct(gpu_lib), problem, grad, kk, xs, src, sstr, nrm, dip,
                       dstr, nq, xt, field0, fstr)
    ref = _call_direct(_bind_direct(reference.lib), problem, grad, kk, xs, src, sstr, nrm,
                       dip, dstr, nq, xt, field0, fstr)
    assert rel_l2(got, ref) < TOL_DIRECT, rel_l2(got, ref)
    assert rel_max(got - field0, ref - field0) < 1e-11


def _dipole_problem(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = W.Problem(name, int(z["problem"]), int(z["depth"]), list(z["order_s"]),
                  list(z["order_r"]), float(z["k"]), z["xs"], z["q"], z["xt"],
                  normals=z["normals"], dipoles=z["dipoles"])
    p.x0, p.D = z["x0"], float(z["D"])
    return p, z


def _fmm(p, xt, precision=engine.FP64):
    cfg = engine.SolverConfig.from_problem(p, precision, engine.POTENTIAL | engine.GRADIENT)
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs, p.normals).set_strengths(p.q, p.dipoles).set_targets(xt).run()
        return s.field()


@pytest.mark.parametrize("name", ["helmholtz_dipole_small", "laplace_dipole_small"])
def test_dipole_gradient(gpu_lib, name):
    """Monopole + dipole sources (the benchmark's sphere configuration has
    them).  (1) The FMM potential equals the reference FMM's (1e-10).
    (2) The FMM gradient is the central difference of the FMM potential,
    on targets whose six shifted copies stay in the same leaf box (so the
    same local expansion and near field apply): 1e-6 relative.  (3) The
    GPU direct gradient equals the restatement's (1e-12).  (4) The FMM
    gradient is within the truncation error of the direct gradient (the
    potential's error is 2e-4 / 3e-5 at these orders)."""
    p, z = _dipole_problem(name)
    w = 2 if p.problem == HELMHOLTZ else 1
    pot, grad = _fmm(p, p.xt)
    assert rel_l2(pot, z["pot"]) < TOL_FP64
    # (2) finite differences of the FMM potential
    h = 1e-6 * p.D
    nb = 2 ** p.depth
    shifts = [np.zeros(3)] + [s * h * np.eye(3)[a] for a in range(3) for s in (1, -1)]
    boxes = [np.floor((p.xt + d - p.x0) / (p.D / nb)).astype(np.int64) for d in shifts]
    same = np.all([np.all(b == boxes[0], axis=1) for b in boxes[1:]], axis=0)
    keep = np.nonzero(same)[0]
    assert keep.size > 0.9 * p.nt
    xt7 = np.concatenate([p.xt[keep] + d for d in shifts])
    pot7, grad7 = _fmm(p, xt7)
    m = keep.size
    pot7 = pot7.reshape(7, m, w)
    g0 = grad7[:3 * w * m].reshape(m, 3, w)
    fd = np.stack([(pot7[1 + 2 * a] - pot7[2 + 2 * a]) / (2 * h) for a in range(3)], axis=1)
    assert rel_l2(g0, fd) < 1e-6, rel_l2(g0, fd)
    # (3) GPU direct gradient with dipoles against the restatement's
    dpot, dgrad = engine.direct(p.problem, p.xs, p.q, p.xt, k=p.k, normals=p.normals,
                                dipoles=p.dipoles)
    assert rel_l2(dpot, z["direct_pot"]) < TOL_DIRECT
    assert rel_l2(dgrad, z["direct_grad"]) < TOL_DIRECT
    # (4) truncation error of the FMM gradient
    e_pot = rel_l2(pot, z["direct_pot"])
    e_grad = rel_l2(grad, z["direct_grad"])
    assert e_grad < 20 * max(e_pot, 1e-8), (e_pot, e_grad)
    assert e_grad < (2e-3 if p.problem == HELMHOLTZ else 5e-4)


def test_helmholtz_1e6_depth6_matches_reference(gpu_lib, reference):
    """The benchmark's Helmholtz cube at full size: 1e6 sources, complex
    strengths, k = 8, depth 6, per-level orders [14, 10, 8, 6, 6, 6],
    targets = sources.  The plain FP64 form equals the reference CPU FMM
    (1e-10, potential and gradient); the FP32 form is within 1e-5 of it
    (its own rounding; both are 6e-5 from the direct sum by truncation)."""
    p = W.helmholtz_cube(1_000_000, k=8.0, depth=6, seed=2)
    nthreads = min(os.cpu_count() or 1, 16)
    r = reference.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs, p.q,
                      p.xt, k=p.k, nthreads=nthreads)
    pot, grad = _fmm(p, p.xt)
    assert rel_l2(pot, r["pot"]) < TOL_FP64
    assert rel_l2(grad, r["grad"]) < TOL_FP64
    assert rel_max(pot, r["pot"]) < TOL_FP64
    pot32, grad32 = _fmm(p, p.xt, engine.FP32)
    assert rel_l2(pot32, pot) < 1e-5
    assert rel_l2(grad32, grad) < 1e-5
