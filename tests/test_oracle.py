"""Pinning of the CPU restatement oracle (no GPU needed).

The restatement (oracle/wbfmm_oracle.c) is checked bit-exactly against the
golden fixtures made by the unmodified reference, and -- where the reference
library is built -- against it live: Morton keys, the stable point sort
`t->ip`, every box {i, n} (with the values the reference's refinement leaves
in non-leaf levels), target boxes, neighbour lists and list-4 interaction
lists with their shift indices (the structural checks of the reference's
neighbour_test / ilist4_test, tools/wbfmm-tests.c.in:1905-2080).  The FP64
direct sums match the reference's direct.c / direct-laplace.c.
"""
import glob
import os

import numpy as np
import pytest

from oracle.oracle_api import HELMHOLTZ, LAPLACE, level_box_offsets
from wbfmm_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not os.path.basename(p).startswith(("dropin_", "direct_")))


@pytest.mark.parametrize("path", CASES, ids=lambda x: os.path.basename(x)[:-4])
def test_tree_matches_golden(restatement, path):
    z = np.load(path)
    ip, boxes = restatement.tree_build(z["x0"], float(z["D"]), int(z["depth"]), z["xs"])
    assert np.array_equal(ip, z["ip"])
    assert np.array_equal(boxes, z["boxes"])


def test_tree_matches_reference_live(restatement, reference):
    for seed, n, depth in [(5, 5000, 4), (6, 333, 3), (7, 20000, 5)]:
        rng = np.random.default_rng(seed)
        xs = rng.uniform(-0.5, 0.5, (n, 3))
        # clustered points exercise empty boxes and the refinement quirks
        xs[: n // 2] = 0.1 * xs[: n // 2] + 0.2
        x0, D = W.fit_box(xs)
        q = rng.standard_normal(n)
        r = reference.fmm(LAPLACE, depth, [0] + [2] * depth, [0] + [2] * depth, x0, D,
                          xs, q, xs[:10], pot=True, grad=False, want_tree=True)
        ip, boxes = restatement.tree_build(x0, D, depth, xs)
        assert np.array_equal(ip, r["ip"])
        assert np.array_equal(boxes, r["boxes"])


def test_point_keys_and_boxes(restatement, reference):
    rng = np.random.default_rng(9)
    x0 = np.array([-0.51, -0.52, -0.5])
    D = 1.03
    for _ in range(2000):
        x = x0 + rng.uniform(0, D, 3)
        assert restatement.point_index_3d(x, x0, D) == reference.point_index_3d(x, x0, D)
        for lv in (1, 3, 6):
            assert restatement.point_box(x0, D, lv, x) == reference.point_box(x0, D, lv, x)
    # box faces, where the floor rule and the truncation rule can differ
    for lv in (2, 4):
        wb = D / 2 ** lv
        for i in range(2 ** lv):
            x = x0 + np.array([i * wb, 0.5 * D, 0.25 * D])
            assert restatement.point_box(x0, D, lv, x) == reference.point_box(x0, D, lv, x)


@pytest.mark.parametrize("level", [2, 3, 4])
def test_neighbour_and_list4(restatement, reference, level):
    nb = 8 ** level
    rng = np.random.default_rng(level)
    boxes = np.unique(np.concatenate([np.arange(min(nb, 64)), rng.integers(0, nb, 200)]))
    for b in boxes:
        b = int(b)
        a = restatement.neighbours(level, b)
        r = reference.neighbours(level, b)
        assert np.array_equal(a, r)
        l4 = restatement.interaction_list_4(level, b)
        r4 = reference.interaction_list_4(level, b)
        assert np.array_equal(l4, r4)
        assert len(l4) <= 189


def test_list4_structure(restatement):
    """ilist4_test semantics: every entry non-adjacent, its parent adjacent
    to ours, shift index = (di+3)*49+(dj+3)*7+dk+3."""
    from wbfmm_b200.engine import HELMHOLTZ as _  # noqa: F401  (package import)

    def decode(m):
        c = [0, 0, 0]
        for b in range(21):
            for a in range(3):
                c[a] |= ((m >> (3 * b + a)) & 1) << b
        return c

    level = 4
    for b in range(0, 8 ** level, 37):
        i = decode(b)
        for s, sh in restatement.interaction_list_4(level, b):
            j = decode(int(s))
            d = [j[a] - i[a] for a in range(3)]
            assert max(abs(x) for x in d) >= 2
            assert max(abs((j[a] >> 1) - (i[a] >> 1)) for a in range(3)) <= 1
            assert sh == (d[0] + 3) * 49 + (d[1] + 3) * 7 + d[2] + 3


@pytest.mark.parametrize("problem", [LAPLACE, HELMHOLTZ])
def test_direct_sum_matches_reference(restatement, reference, problem):
    rng = np.random.default_rng(31)
    xs = rng.uniform(-0.5, 0.5, (3000, 3))
    xt = rng.uniform(-0.5, 0.5, (40, 3))
    q = rng.standard_normal(3000 * (2 if problem == HELMHOLTZ else 1))
    k = 5.0
    pot, grad = restatement.direct(problem, xs, q, xt, k=k)
    rp = reference.direct(problem, xs, q, xt, k=k, grad=False)
    rg = reference.direct(problem, xs, q, xt, k=k, grad=True)
    assert np.max(np.abs(pot - rp)) / np.max(np.abs(rp)) < 1e-13
    assert np.max(np.abs(grad - rg)) / np.max(np.abs(rg)) < 1e-13


def test_direct_sum_dipoles_match_reference(restatement, reference):
    rng = np.random.default_rng(32)
    xs = rng.uniform(-0.5, 0.5, (2000, 3))
    nrm = rng.standard_normal((2000, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    xt = rng.uniform(-0.5, 0.5, (30, 3))
    q = rng.standard_normal(4000)
    d = rng.standard_normal(4000)
    pot, _ = restatement.direct(HELMHOLTZ, xs, q, xt, k=3.0, normals=nrm, dipoles=d,
                                grad=False)
    ref = reference.direct(HELMHOLTZ, xs, q, xt, k=3.0, normals=nrm, dipoles=d)
    assert np.max(np.abs(pot - ref)) / np.max(np.abs(ref)) < 1e-13


def test_dipole_gradient_by_finite_differences(restatement):
    """Dipole gradients have no reference counterpart (the reference aborts,
    src/local.c:259, src/direct.c:223): pin the oracle's analytic gradient
    with central differences of the reference-supported potential."""
    rng = np.random.default_rng(33)
    xs = rng.uniform(-0.5, 0.5, (50, 3))
    nrm = rng.standard_normal((50, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    xt = rng.uniform(-0.5, 0.5, (5, 3))
    h = 1e-5
    for problem, w in ((HELMHOLTZ, 2), (LAPLACE, 1)):
        q = rng.standard_normal(50 * w)
        d = rng.standard_normal(50 * w)
        _, g = restatement.direct(problem, xs, q, xt, k=4.0, normals=nrm, dipoles=d)
        g = g.reshape(5, 3, w)
        for a in range(3):
            e = np.zeros(3); e[a] = h
            pp, _ = restatement.direct(problem, xs, q, xt + e, k=4.0, normals=nrm,
                                       dipoles=d, grad=False)
            pm, _ = restatement.direct(problem, xs, q, xt - e, k=4.0, normals=nrm,
                                       dipoles=d, grad=False)
            fd = ((pp - pm) / (2 * h)).reshape(5, w)
            assert np.allclose(g[:, a, :], fd, rtol=1e-5, atol=1e-6 * np.abs(fd).max())


def test_golden_direct_sums(restatement):
    z = np.load(os.path.join(GOLDEN, "helmholtz_small.npz"))
    pot, grad = restatement.direct(HELMHOLTZ, z["xs"], z["q"], z["xt"][:50], k=float(z["k"]))
    assert np.allclose(pot, z["direct_pot"][:100], rtol=0, atol=1e-12 * np.abs(pot).max())


def test_box_offsets():
    assert level_box_offsets(2) == [0, 1, 9, 73]


def test_curl_convention_matches_reference(restatement, reference):
    """The Laplace curl as e_ijk d_j A_k of the three components' direct
    gradients (how the engine forms it) is the reference's direct curl
    (WBFMM_FIELD_CURL with three source components)."""
    from oracle.oracle_api import curl_from_gradients
    rng = np.random.default_rng(61)
    xs = rng.uniform(-0.5, 0.5, (300, 3))
    xt = rng.uniform(-0.5, 0.5, (40, 3))
    q3 = rng.standard_normal((300, 3))
    g = [restatement.direct(LAPLACE, xs, q3[:, c].copy(), xt, pot=False, grad=True)[1]
         for c in range(3)]
    mine = curl_from_gradients(g)
    ref = reference.direct_curl(xs, q3, xt)
    assert np.linalg.norm(mine - ref) <= 1e-12 * np.linalg.norm(ref)


def test_curl_gradient_convention_matches_reference(reference):
    """The reference's direct curl gradient (WBFMM_FIELD_CURL |
    WBFMM_FIELD_GRADIENT): the curl, then d/dx, d/dy, d/dz of its three
    components, formed here from the second derivatives of 1/(4 pi r) as the
    engine combines them (curl_i = e_ijk d_j A_k; entry 3 + 3 a + i is
    d_a curl_i)."""
    rng = np.random.default_rng(67)
    xs = rng.uniform(-0.5, 0.5, (200, 3))
    xt = rng.uniform(-0.5, 0.5, (30, 3))
    q3 = rng.standard_normal((200, 3))
    d = xt[:, None, :] - xs[None, :, :]
    r = np.linalg.norm(d, axis=2)
    g = -d / (4 * np.pi * r[..., None] ** 3)                       # d_j (1/4 pi r)
    H = (3 * d[..., :, None] * d[..., None, :] / r[..., None, None] ** 2
         - np.eye(3)) / (4 * np.pi * r[..., None, None] ** 3)     # d_a d_j (1/4 pi r)
    G = np.einsum("tsj,sc->tcj", g, q3)                            # d_j A_c
    HH = np.einsum("tsaj,sc->tcaj", H, q3)                         # d_a d_j A_c
    curl = np.stack([G[:, 2, 1] - G[:, 1, 2], G[:, 0, 2] - G[:, 2, 0],
                     G[:, 1, 0] - G[:, 0, 1]], axis=1)
    dcurl = np.stack([HH[:, 2, :, 1] - HH[:, 1, :, 2], HH[:, 0, :, 2] - HH[:, 2, :, 0],
                      HH[:, 1, :, 0] - HH[:, 0, :, 1]], axis=2)    # [t, a, i]
    mine = np.hstack([curl, dcurl.reshape(-1, 9)])
    ref = reference.direct_curl_gradient(xs, q3, xt)
    assert np.linalg.norm(mine - ref) <= 1e-12 * np.linalg.norm(ref)


def test_reference_local_curl_gradient_is_inexact(reference):
    """The reference's evaluation of the curl gradient from a local
    expansion (wbfmm_laplace_expansion_local_eval, WBFMM_FIELD_CURL |
    WBFMM_FIELD_GRADIENT, src/local-laplace.c:752-1010) is not the derivative
    of its curl evaluation (WBFMM_FIELD_CURL, :632-750): central differences
    of the curl differ from it by far more than their own error on random
    order-10 coefficients.  The engine evaluates the exact derivative
    (derived expansions through the gradient L2P), so curl-gradient parity is
    measured against the reference's direct sums."""
    import ctypes as C
    f = reference.lib.wbfmm_laplace_expansion_local_eval
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint, C.c_void_p,
                  C.c_void_p, C.c_int, C.c_void_p]
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    N, nq = 10, 3
    rng = np.random.default_rng(5)
    cf = rng.standard_normal((N + 1) ** 2 * nq)
    x0, work = np.zeros(3), np.zeros(100000)

    def ev(field, x, nout):
        out, xf = np.zeros(nout), np.array(x, dtype=float)
        f(ptr(x0), ptr(cf), nq, N, nq, field, ptr(xf), ptr(out), 1, ptr(work))
        return out
    worst = 0.0
    for _ in range(5):
        x = rng.uniform(-0.3, 0.3, 3)
        cg = ev(4 | 2, x, 12)
        assert np.array_equal(cg[:3], ev(4, x, 3))
        for a in range(3):
            e = 1e-5
            xp, xm = x.copy(), x.copy()
            xp[a] += e; xm[a] -= e
            fd = (ev(4, xp, 3) - ev(4, xm, 3)) / (2 * e)
            worst = max(worst, np.abs(fd - cg[3 + 3 * a:6 + 3 * a]).max() / np.abs(cg[3:]).max())
    assert worst > 1e-5, worst


DIRECT_CASES = ("helm_mono", "helm_mixed", "lap_mono", "lap_dipole", "lap_mixed")


def direct_case(name):
    """Inputs and the reference's outputs of one case of direct_sums.npz
    (the reference's own direct sums, make_direct_golden.py)."""
    z = np.load(os.path.join(GOLDEN, "direct_sums.npz"))

    def g(a):
        v = z[f"{name}_{a}"]
        return v if v.size else None

    return {a: g(a) for a in ("xs", "xt", "q", "normals", "dipoles", "pot")} | {
        "problem": int(z[f"{name}_problem"]), "k": float(z[f"{name}_k"]),
        "grad": g("grad") if f"{name}_grad" in z.files else None}


@pytest.mark.parametrize("name", DIRECT_CASES)
def test_restatement_direct_matches_reference_fixture(restatement, name):
    """The restatement's direct sums equal the reference's (src/direct.c,
    src/direct-laplace.c) to 1e-13.  For Laplace monopoles plus dipoles the
    reference leaves the 1/(4 pi) off the dipole term
    (src/direct-laplace.c:261-263), the restatement (like the FMM) does not:
    there the reference's value is the monopole sum plus 4 pi times the
    dipole sum."""
    c = direct_case(name)
    kw = dict(k=c["k"], normals=c["normals"], dipoles=c["dipoles"])
    pot, grad = restatement.direct(c["problem"], c["xs"], c["q"], c["xt"], **kw)
    if name == "lap_mixed":
        mono, _ = restatement.direct(c["problem"], c["xs"], c["q"], c["xt"], grad=False)
        dip, _ = restatement.direct(c["problem"], c["xs"], None, c["xt"], grad=False, **kw)
        pot = mono + 4.0 * np.pi * dip
    assert np.linalg.norm(pot - c["pot"]) <= 1e-13 * np.linalg.norm(c["pot"])
    if c["grad"] is not None:
        assert np.linalg.norm(grad - c["grad"]) <= 1e-13 * np.linalg.norm(c["grad"])
