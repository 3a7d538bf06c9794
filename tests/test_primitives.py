"""The single-expansion primitives of the drop-in (wbfmm_b200/csrc/primitives.cu)
against the reference library's own (oracle/_ref/libwbfmm_ref.so) on the
same inputs: expansion coefficients of a source, evaluation of regular and
singular expansions, rotation and coaxial tables, rotation and coaxial
translation of one expansion (src/wbfmm.h:247-420, :525-643), and the
scalar helpers.  The array primitives run on the GPU; the scalar helpers
are checked on the CPU."""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "wbfmm_b200", "libwbfmm_b200.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libwbfmm_ref.so")

D, I, U, VP = C.c_double, C.c_int, C.c_uint, C.c_void_p


def _libs():
    if not os.path.exists(REF):
        pytest.skip("reference library not built (needs the reference sources)")
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    return C.CDLL(LIB), C.CDLL(REF)


def _p(a):
    return a.ctypes.data_as(VP)


def _nrot(N):
    # entries n <= N of a rotation table: rot_idx(N+1, 0, N+1), the count the
    # reference copies out (src/rotations.c:200)
    n = N + 1
    return n * (4 * n - 1) * (n + 1) // 6 + 2 * n * (n + 1)


def _ncoax(L):
    return (L + 1) * (L + 2) * (L + 3) // 6 + (L + 1) * (L + 2) // 2 + L + 1


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


SIGS = {
    "wbfmm_coefficients_H_rotation": [VP, I, D, VP],
    "wbfmm_coefficients_RR_coaxial": [VP, I, D, VP],
    "wbfmm_coefficients_SR_coaxial": [VP, I, D, VP],
    "wbfmm_rotate_H_ref": [VP, I, VP, I, I, I, VP, D, D, D],
    "wbfmm_laplace_rotate_H_ref": [VP, I, VP, I, I, I, VP, D, D, D],
    "wbfmm_coaxial_translate_ref": [VP, I, I, VP, I, I, I, VP, I, I, D],
    "wbfmm_laplace_coaxial_translate_SS": [VP, I, I, VP, I, I, I, D, D],
    "wbfmm_laplace_coaxial_translate_RR": [VP, I, I, VP, I, I, I, D, D],
    "wbfmm_laplace_coaxial_translate_SR": [VP, I, I, VP, I, I, I, D, D],
    "wbfmm_laplace_coaxial_translate_init": [I],
    "wbfmm_expansion_h_cfft": [D, I, VP, VP, VP, I, VP, I, VP],
    "wbfmm_expansion_j_evaluate": [D, VP, VP, I, I, I, VP, VP, I, VP],
    "wbfmm_expansion_h_evaluate": [D, VP, VP, I, I, I, VP, VP, I, VP],
    "wbfmm_laplace_expansion_cfft": [I, VP, VP, VP, I, VP, I, VP],
    "wbfmm_laplace_expansion_evaluate": [VP, VP, I, I, I, VP, VP, VP],
    "wbfmm_laplace_expansion_local_eval": [VP, VP, I, I, I, U, VP, VP, I, VP],
    "wbfmm_legendre_init": [D, D, VP, VP, VP],
    "wbfmm_bessel_j_init": [D, VP, VP],
    "wbfmm_bessel_j_recursion": [VP, VP, D, I],
    "wbfmm_bessel_h_init": [D, VP, VP],
    "wbfmm_bessel_h_recursion": [VP, VP, D, I],
    "wbfmm_cartesian_to_spherical": [VP, VP, VP, VP, VP],
}


def _fn(lib, name):
    f = getattr(lib, name)
    f.argtypes = SIGS[name]
    f.restype = I
    return f


@pytest.fixture(scope="module")
def libs():
    return _libs()


def both(libs, name, args_fn):
    """Call `name` in the drop-in and the reference with fresh copies of the
    arrays made by args_fn(); return both argument lists."""
    out = []
    for lib in libs:
        args = args_fn()
        _fn(lib, name)(*[(_p(a) if isinstance(a, np.ndarray) else a) for a in args])
        out.append(args)
    return out


def test_scalar_helpers(libs):
    """Legendre and Bessel starting values and recursions, spherical
    coordinates: the same routines on the host."""
    mine, ref = libs
    rng = np.random.default_rng(1)
    for _ in range(20):
        x0, x = rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3)
        a = [np.zeros(1) for _ in range(3)]
        b = [np.zeros(1) for _ in range(3)]
        _fn(mine, "wbfmm_cartesian_to_spherical")(_p(x0), _p(x), *map(_p, a))
        _fn(ref, "wbfmm_cartesian_to_spherical")(_p(x0), _p(x), *map(_p, b))
        assert np.allclose(np.concatenate(a), np.concatenate(b), rtol=1e-15, atol=1e-15)
        C_, S_ = np.cos(a[1][0]), np.sin(a[1][0])
        p = [np.zeros(1) for _ in range(3)]
        q = [np.zeros(1) for _ in range(3)]
        _fn(mine, "wbfmm_legendre_init")(C_, S_, *map(_p, p))
        _fn(ref, "wbfmm_legendre_init")(C_, S_, *map(_p, q))
        assert np.allclose(np.concatenate(p), np.concatenate(q), rtol=1e-15, atol=0)
        xb = rng.uniform(0.05, 20.0)
        for init, rec, w in (("wbfmm_bessel_j_init", "wbfmm_bessel_j_recursion", 1),
                             ("wbfmm_bessel_h_init", "wbfmm_bessel_h_recursion", 2)):
            vals = []
            for lib in libs:
                j0, j1 = np.zeros(w), np.zeros(w)
                _fn(lib, init)(xb, _p(j0), _p(j1))
                seq = [j0.copy(), j1.copy()]
                for n in range(1, 12):
                    _fn(lib, rec)(_p(j0), _p(j1), xb, n)
                    seq.append(j1.copy())
                vals.append(np.concatenate(seq))
            assert _rel(vals[0], vals[1]) < 1e-12, (init, xb)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [1, 6, 15])
def test_rotation_and_coaxial_tables(gpu_lib, libs, N):
    a, b = both(libs, "wbfmm_coefficients_H_rotation",
                lambda: [np.zeros(_nrot(N) + 8), N, 0.7321, np.zeros(100000)])
    n = _nrot(N)
    # the rotation recursion (G&D 5.55) grows rounding differences with the
    # degree (FMA contraction on the GPU against the reference's sequence)
    assert _rel(a[0][:n], b[0][:n]) < (1e-13 if N <= 8 else 1e-8)
    for name, nc in (("wbfmm_coefficients_RR_coaxial", 1), ("wbfmm_coefficients_SR_coaxial", 2)):
        for kr in (0.37, 4.2, 15.0):
            a, b = both(libs, name, lambda: [np.zeros(nc * _ncoax(N) + 16), N, kr, np.zeros(100000)])
            # entries l <= N of both tables
            m = nc * (N * (N + 1) * (N + 2) // 6 + N * (N + 1) // 2 + N + 1)
            assert _rel(a[0][:m], b[0][:m]) < 1e-12, (name, kr)


@pytest.mark.gpu
@pytest.mark.parametrize("helm", [True, False])
def test_expansion_of_a_source_and_its_evaluation(gpu_lib, libs, helm):
    """Expansion coefficients of two sources (three components, strided)
    added to existing ones, then the singular and regular evaluations."""
    rng = np.random.default_rng(2)
    N, nq, cstr = 12, 3, 4
    w = 2 if helm else 1
    nc = (N + 1) ** 2
    c0 = rng.standard_normal(w * nc * cstr)
    x0 = np.array([0.1, -0.2, 0.05])
    xs = [x0 + rng.uniform(-0.3, 0.3, 3) for _ in range(2)]
    qs = [rng.standard_normal(w * nq) for _ in range(2)]

    def run(lib):
        c = c0.copy()
        for x, q in zip(xs, qs):
            if helm:
                _fn(lib, "wbfmm_expansion_h_cfft")(2.5, N, _p(x0), _p(x), _p(q), nq, _p(c), cstr,
                                                  _p(np.zeros(100000)))
            else:
                _fn(lib, "wbfmm_laplace_expansion_cfft")(N, _p(x0), _p(x), _p(q), nq, _p(c), cstr,
                                                        _p(np.zeros(100000)))
        return c
    ca, cb = run(libs[0]), run(libs[1])
    assert _rel(ca, cb) < 1e-13
    for k_ev in range(2):
        for xf in (x0 + np.array([1.3, 0.7, -0.9]), x0 + np.array([0.02, -0.05, 0.03])):
            outs = []
            for lib in libs:
                if helm:
                    fstr = 3
                    f = np.full(fstr * nq, 0.25)
                    name = "wbfmm_expansion_h_evaluate" if k_ev == 0 else "wbfmm_expansion_j_evaluate"
                    _fn(lib, name)(2.5, _p(x0), _p(cb), cstr, N, nq, _p(xf), _p(f), fstr,
                                   _p(np.zeros(100000)))
                elif k_ev == 0:
                    f = np.full(nq, 0.25)
                    _fn(lib, "wbfmm_laplace_expansion_evaluate")(_p(x0), _p(cb), cstr, N, nq, _p(xf),
                                                                 _p(f), _p(np.zeros(100000)))
                else:
                    f = np.full(nq, 0.25)
                    _fn(lib, "wbfmm_laplace_expansion_local_eval")(_p(x0), _p(cb), cstr, N, nq, 1,
                                                                   _p(xf), _p(f), 1, _p(np.zeros(100000)))
                    g = np.full(3 * nq, -0.5)
                    _fn(lib, "wbfmm_laplace_expansion_local_eval")(_p(x0), _p(cb), cstr, N, nq, 2,
                                                                   _p(xf), _p(g), 3, _p(np.zeros(100000)))
                    f = np.concatenate([f, g])
                outs.append(f)
            assert _rel(outs[0], outs[1]) < 1e-12, (helm, k_ev, xf)


@pytest.mark.gpu
@pytest.mark.parametrize("helm", [True, False])
def test_rotation_of_an_expansion(gpu_lib, libs, helm):
    rng = np.random.default_rng(3)
    N, nq, cstri, cstro = 14, 2, 3, 2
    w = 2 if helm else 1
    nc = (N + 1) ** 2
    H = np.zeros(_nrot(N) + 8)
    _fn(libs[1], "wbfmm_coefficients_H_rotation")(_p(H), N, 1.1, _p(np.zeros(100000)))
    Ci = rng.standard_normal(w * nc * cstri)
    Co0 = rng.standard_normal(w * nc * cstro)
    name = "wbfmm_rotate_H_ref" if helm else "wbfmm_laplace_rotate_H_ref"
    for sc in (0.0, 1.0, -0.5):
        a, b = both(libs, name, lambda: [Co0.copy(), cstro, Ci.copy(), cstri, N, nq, H.copy(),
                                         0.4, -1.3, sc])
        assert _rel(a[0], b[0]) < 1e-12, sc


@pytest.mark.gpu
def test_helmholtz_coaxial_translation(gpu_lib, libs):
    rng = np.random.default_rng(4)
    L, nq, cstri, cstro = 16, 2, 2, 3
    for name_t, cplx in (("wbfmm_coefficients_SR_coaxial", 1), ("wbfmm_coefficients_RR_coaxial", 0)):
        tab = np.zeros((2 if cplx else 1) * _ncoax(L) + 16)
        _fn(libs[1], name_t)(_p(tab), L, 3.7, _p(np.zeros(100000)))
        # No <= Ni: for output degrees above Ni + 1 the reference reads input
        # degrees up to No - 1, beyond the input expansion
        # (src/translations.c:455-462); the drop-in sums degrees <= Ni
        for No, Ni in ((12, 12), (10, 14), (15, 15)):
            Ci = rng.standard_normal(2 * (Ni + 1) ** 2 * cstri)
            Co0 = rng.standard_normal(2 * (No + 1) ** 2 * cstro)
            for sc in (0.0, 1.0):
                a, b = both(libs, "wbfmm_coaxial_translate_ref",
                            lambda: [Co0.copy(), cstro, No, Ci.copy(), cstri, Ni, nq, tab.copy(), L,
                                     cplx, sc])
                assert np.all(np.isfinite(a[0])) and np.all(np.isfinite(b[0])), (
                    np.flatnonzero(~np.isfinite(a[0]))[:8], np.flatnonzero(~np.isfinite(b[0]))[:8])
                assert _rel(a[0], b[0]) < 1e-12, (name_t, No, Ni, sc)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["SS", "RR", "SR"])
def test_laplace_coaxial_translation(gpu_lib, libs, kind):
    rng = np.random.default_rng(5)
    _fn(libs[1], "wbfmm_laplace_coaxial_translate_init")(40)
    nq, cstri, cstro = 2, 2, 3
    name = "wbfmm_laplace_coaxial_translate_" + kind
    cases = ((10, 10), (8, 12), (12, 8))
    if kind == "RR":
        # the reference's R|R forms powers of t only up to Ni + 1 and writes
        # m = 0 outputs up to degree Ni whatever No (src/laplace.c:600-610):
        # compared where both are defined
        cases = ((10, 10), (11, 10))
    for No, Ni in cases:
        nin = max(No, Ni) if kind == "RR" else Ni
        Ci = rng.standard_normal((nin + 1) ** 2 * cstri)
        Co0 = rng.standard_normal((No + 1) ** 2 * cstro)
        for t in (0.75, -1.5):
            for sc in (0.0, 1.0, 0.5):
                a, b = both(libs, name, lambda: [Co0.copy(), cstro, No, Ci.copy(), cstri, Ni, nq,
                                                 t, sc])
                assert _rel(a[0], b[0]) < 1e-12, (kind, No, Ni, t, sc)
