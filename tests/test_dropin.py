"""The drop-in wbfmm.h API (include/wbfmm.h over libwbfmm_b200.so).

A wbfmm client program (tests/dropin/driver.c), written only against the
wbfmm.h API in the reference drivers' call order
(tools/wbfmm-tree-calc.c.in:262-414, tools/wbfmm-laplace-tree-calc.c.in:
336-460), is compiled against include/wbfmm.h and run on the GPU; what it
sees -- fields, t->ip, every box's {i, n}, the coefficient arrays behind
t->mps / t->mpr -- must equal what the same program sees against the
reference (tests/golden/dropin_cases.npz, made by
tests/golden/make_dropin_golden.py; and the live reference build of the
program where it exists).  FP64 tolerance: 1e-10 relative.

The host-only parts of the API (indexing, neighbour and interaction lists,
truncation numbers, configuration) run without a GPU and are checked here
against the reference and the CPU restatement.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "dropin"))

import harness as H  # noqa: E402

GOLDEN = os.path.join(HERE, "golden", "dropin_cases.npz")
LIB = os.path.join(ROOT, "wbfmm_b200", "libwbfmm_b200.so")
TOL = 1e-10

_u64p = C.POINTER(C.c_uint64)
_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib():
    lib = C.CDLL(LIB)
    lib.wbfmm_box_index.restype = C.c_uint64
    lib.wbfmm_box_index.argtypes = [C.c_uint32] * 3
    lib.wbfmm_box_location.argtypes = [C.c_uint64] + [C.POINTER(C.c_uint32)] * 3
    lib.wbfmm_box_parent.restype = C.c_uint64
    lib.wbfmm_box_parent.argtypes = [C.c_uint64]
    lib.wbfmm_box_first_child.restype = C.c_uint64
    lib.wbfmm_box_first_child.argtypes = [C.c_uint64]
    lib.wbfmm_point_index_3d.restype = C.c_uint64
    lib.wbfmm_point_index_3d.argtypes = [_dp, _dp, C.c_double]
    lib.wbfmm_point_locate_box.restype = C.c_uint64
    lib.wbfmm_point_locate_box.argtypes = [C.c_uint64, C.c_uint]
    lib.wbfmm_box_neighbours.argtypes = [C.c_uint, C.c_uint64, _u64p]
    lib.wbfmm_box_interaction_list_4.argtypes = [C.c_uint, C.c_uint64, _u64p, C.c_int]
    lib.wbfmm_box_interaction_grid_4.argtypes = [C.c_uint, C.c_uint64, _u64p]
    lib.wbfmm_box_location_from_index.argtypes = [C.c_uint64, C.c_uint32, _dp,
                                                  C.c_double, _dp, _dp]
    lib.wbfmm_tree_new.restype = C.c_void_p
    lib.wbfmm_tree_new.argtypes = [_dp, C.c_double, C.c_uint]
    lib.wbfmm_tree_box_centre.argtypes = [C.c_void_p, C.c_uint, C.c_uint64, _dp, _dp]
    lib.wbfmm_truncation_number.argtypes = [C.c_void_p, C.c_double, C.c_uint, C.c_double]
    lib.wbfmm_points_origin_width.argtypes = [_dp, C.c_int, C.c_int, _dp, _dp, _dp,
                                              C.c_int]
    return lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


# ------------------------------------------------------------ host side
def test_box_index_roundtrip(lib):
    rng = np.random.default_rng(1)
    for i, j, k in rng.integers(0, 1 << 20, (200, 3)):
        b = lib.wbfmm_box_index(int(i), int(j), int(k))
        x, y, z = C.c_uint32(), C.c_uint32(), C.c_uint32()
        lib.wbfmm_box_location(b, C.byref(x), C.byref(y), C.byref(z))
        assert (x.value, y.value, z.value) == (i, j, k)
        assert lib.wbfmm_box_parent(b) == b >> 3
        assert lib.wbfmm_box_first_child(b) == b << 3


def test_point_index_matches_restatement(lib, restatement):
    rng = np.random.default_rng(2)
    x0 = np.array([-1.0, -0.5, -2.0])
    D = 3.0
    pts = x0 + rng.uniform(0, D, (300, 3))
    ours = [lib.wbfmm_point_index_3d(_p(np.ascontiguousarray(p)), _p(x0), D) for p in pts]
    theirs = [restatement.point_index_3d(p, x0, D) for p in pts]
    assert ours == theirs
    for level in (1, 4, 9):
        for m in ours[:20]:
            assert lib.wbfmm_point_locate_box(m, level) == m >> (3 * (20 - level))


@pytest.mark.parametrize("level", [2, 3, 4])
def test_neighbours_and_list4_match_restatement(lib, restatement, level):
    nb = np.zeros(27, np.uint64)
    l4 = np.zeros(2 * 189, np.uint64)
    grid = np.zeros(343, np.uint64)
    for b in range(0, 8 ** level, max(1, 8 ** level // 97)):
        n = lib.wbfmm_box_neighbours(level, b, _p(nb, _u64p))
        assert sorted(nb[:n].tolist()) == sorted(restatement.neighbours(level, b).tolist())
        n = lib.wbfmm_box_interaction_list_4(level, b, _p(l4, _u64p), 0)
        ours = [(int(l4[2 * i]), int(l4[2 * i + 1])) for i in range(n)]
        assert ours == [tuple(map(int, e)) for e in restatement.interaction_list_4(level, b)]
        lib.wbfmm_box_interaction_grid_4(level, b, _p(grid, _u64p))
        for s, sh in ours:
            assert grid[sh] == s + 1
        assert np.count_nonzero(grid) == n
        # sorted: the same entries, equal shift directions contiguous
        n2 = lib.wbfmm_box_interaction_list_4(level, b, _p(l4, _u64p), 1)
        srt = [(int(l4[2 * i]), int(l4[2 * i + 1])) for i in range(n2)]
        assert sorted(srt) == sorted(ours)
        dirs = []
        for _, sh in srt:
            d = np.array([sh // 49 - 3, sh // 7 % 7 - 3, sh % 7 - 3], float)
            dirs.append(tuple(np.round(d / np.linalg.norm(d), 12)))
        seen, prev = set(), None
        for d in dirs:
            if d != prev:
                assert d not in seen, "shift directions not grouped"
                seen.add(d)
            prev = d


def test_truncation_number_matches_reference(lib, reference):
    x0 = np.array([0.0, 0.0, 0.0])
    rl = reference.lib
    rl.wbfmm_tree_new.restype = C.c_void_p
    rl.wbfmm_tree_new.argtypes = [_dp, C.c_double, C.c_uint]
    rl.wbfmm_truncation_number.argtypes = [C.c_void_p, C.c_double, C.c_uint, C.c_double]
    for D in (1.0, 2.5):
        ours = lib.wbfmm_tree_new(_p(x0), D, 8)
        theirs = rl.wbfmm_tree_new(_p(x0), D, 8)
        for k in (0.5, 4.0, 20.0):
            for level in range(1, 8):
                for tol in (1e-3, 1e-6, 1e-10):
                    assert (lib.wbfmm_truncation_number(ours, k, level, tol) ==
                            rl.wbfmm_truncation_number(theirs, k, level, tol))


def test_box_geometry_and_origin_width(lib):
    x0 = np.array([-1.0, 2.0, 0.5])
    D = 4.0
    t = lib.wbfmm_tree_new(_p(x0), D, 8)
    xb, wb = np.zeros(3), np.zeros(1)
    b = lib.wbfmm_box_index(2, 3, 1)
    lib.wbfmm_tree_box_centre(t, 2, b, _p(xb), _p(wb))
    assert wb[0] == 1.0 and np.allclose(xb, x0 + np.array([2.5, 3.5, 1.5]))
    lib.wbfmm_box_location_from_index(b, 2, _p(x0), D, _p(xb), _p(wb))
    assert np.allclose(xb, x0 + np.array([2.0, 3.0, 1.0]))
    pts = np.random.default_rng(3).uniform(-3, 5, (100, 4))
    lo, hi, w = np.zeros(3), np.zeros(3), np.zeros(1)
    lib.wbfmm_points_origin_width(_p(pts), 4, 100, _p(lo), _p(hi), _p(w), 1)
    assert np.array_equal(lo, pts[:, :3].min(0)) and np.array_equal(hi, pts[:, :3].max(0))
    assert w[0] == (hi - lo).max()


def test_client_program_compiles_against_dropin_header():
    assert os.path.exists(H.build_driver("b200"))


def test_reference_client_reproduces_golden():
    """Pins the fixture: the live reference build of the client program
    gives the stored outputs."""
    if H.build_driver("reference") is None:
        pytest.skip("reference build of the client program not available")
    g = np.load(GOLDEN)
    for name, c in list(H.cases().items())[:3]:
        _compare(name, c, H.run("reference", c), g, tol=1e-13)


# ------------------------------------------------------------- GPU side
def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _compare(name, c, out, g, tol=TOL):
    f_ref = g[f"{name}/f"]
    assert out["f"].shape == f_ref.shape
    assert _rel(out["f"], f_ref) <= tol, (name, _rel(out["f"], f_ref))
    assert np.abs(out["f"] - f_ref).max() <= 10 * tol * np.abs(f_ref).max()
    assert np.array_equal(out["ip"], g[f"{name}/ip"])
    boxes = np.concatenate([out[f"boxes{l}"] for l in range(c.depth + 1)])
    assert np.array_equal(boxes, g[f"{name}/boxes"])
    rng = np.random.default_rng(7)
    for l in range(1, c.depth + 1):
        for kind in ("mps", "mpr"):
            a = out[f"{kind}{l}"]
            nrm = float(g[f"{name}/{kind}{l}_norm"])
            assert abs(np.linalg.norm(a) - nrm) <= tol * nrm, (name, kind, l)
            proj = np.random.default_rng(7).standard_normal((16, a.size)) @ a
            assert np.abs(proj - g[f"{name}/{kind}{l}_proj"]).max() <= 4 * tol * nrm, (name, kind, l)
    del rng


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(H.cases().keys()))
def test_dropin_client_matches_reference(gpu_lib, name):
    c = H.cases()[name]
    out = H.run("b200", c)
    _compare(name, c, out, np.load(GOLDEN))
    if H.build_driver("reference") is not None:
        ref = H.run("reference", c)
        for l in range(1, c.depth + 1):
            for kind in ("mps", "mpr"):
                a, b = out[f"{kind}{l}"], ref[f"{kind}{l}"]
                assert np.abs(a - b).max() <= TOL * np.abs(b).max(), (name, kind, l)


DRIVER_CASES = [
    ("wbfmm-tree-calc", ["-b", "-d", "3", "-k", "4", "-R", "8", "-S", "8"]),
    ("wbfmm-tree-calc", ["-b", "-d", "3", "-k", "4", "-R", "8", "-S", "8", "-g"]),
    ("wbfmm-tree-calc", ["-b", "-d", "3", "-k", "4", "-t", "1e-6"]),
    ("wbfmm-laplace-tree-calc", ["-b", "-d", "3", "-R", "8", "-S", "8"]),
    ("wbfmm-laplace-tree-calc", ["-b", "-d", "3", "-R", "8", "-S", "8", "-g"]),
    ("wbfmm-laplace-tree-calc", ["-b", "-d", "3", "-R", "8", "-S", "8", "-l"]),
]


def _write_points(path, rows, nq, code):
    with open(path, "w") as f:
        f.write(f"{rows.shape[0]} {nq} {code}\n")
        for r in rows:
            f.write(" ".join("%.17g" % v for v in r) + "\n")


def _read_fields(text):
    return np.array([[float(v) for v in line.split()] for line in text.strip().splitlines()])


@pytest.mark.gpu
@pytest.mark.parametrize("tool,args", DRIVER_CASES, ids=lambda x: x if isinstance(x, str) else " ".join(x))
def test_reference_driver_on_dropin(gpu_lib, tmp_path, tool, args):
    """The reference's own command-line driver (unmodified source, its text
    point files in and fields out), built once against the reference library
    and once against this drop-in: the same output to 1e-10."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", tool + "-reference")
    b200_bin = os.path.join(ROOT, "oracle", "_ref", tool + "-b200")
    if not (os.path.exists(ref_bin) and os.path.exists(b200_bin)):
        pytest.skip("reference drivers not built (needs the reference sources)")
    rng = np.random.default_rng(81)
    n, nf = 3000, 200
    xs = rng.uniform(-0.5, 0.5, (n, 3))
    helm = tool == "wbfmm-tree-calc"
    q = rng.standard_normal((n, 2 if helm else 1))
    _write_points(tmp_path / "src.txt", np.hstack([xs, q]), q.shape[1], "M")
    _write_points(tmp_path / "fld.txt", rng.uniform(-0.5, 0.5, (nf, 3)), 0, "F")
    runs = [subprocess.run([b, "-s", str(tmp_path / "src.txt"), "-f", str(tmp_path / "fld.txt"),
                            *args], capture_output=True, text=True, timeout=300,
                           env=dict(os.environ, MALLOC_MMAP_THRESHOLD_=str(32 << 20)))
            for b in (ref_bin, b200_bin)]
    if helm and "-g" in args:
        # the driver passes field stride 2 with the gradient field; the
        # reference aborts on it (src/local.c:293-296), and so does the drop-in
        for r in runs:
            assert r.returncode != 0 and "too small for gradient" in r.stderr
        return
    for r in runs:
        assert r.returncode == 0, r.stderr[-2000:]
    outs = [_read_fields(r.stdout) for r in runs]
    a, b = outs
    assert a.shape == b.shape and a.shape[0] == nf
    assert np.array_equal(a[:, :3], b[:, :3])
    fa, fb = a[:, 3:], b[:, 3:]
    assert np.linalg.norm(fb - fa) <= 1e-10 * np.linalg.norm(fa)


CURL_DRIVER_CASES = [
    ("wbfmm-laplace-tree-calc", ["-b", "-d", "3", "-R", "8", "-S", "8"]),
    ("wbfmm-laplace-tree-calc", ["-b", "-d", "3", "-R", "8", "-S", "8", "-c"]),
    ("wbfmm-laplace-tree-calc", ["-b", "-d", "3", "-R", "10", "-S", "10", "-c", "-g"]),
    ("wbfmm-laplace-tree-calc-float", ["-b", "-d", "3", "-R", "8", "-S", "8", "-c"]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("tool,args", CURL_DRIVER_CASES, ids=lambda x: x if isinstance(x, str) else " ".join(x))
def test_reference_driver_vector_sources_on_dropin(gpu_lib, tmp_path, tool, args):
    """The reference's Laplace driver on three-component sources (a vector
    potential): the three potentials, the curl (-c) and the curl with its
    gradient (-c -g), through the drop-in's multi-component trees, against
    the same driver built on the reference library."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", tool + "-reference")
    b200_bin = os.path.join(ROOT, "oracle", "_ref", tool + "-b200")
    if not (os.path.exists(ref_bin) and os.path.exists(b200_bin)):
        pytest.skip("reference drivers not built (needs the reference sources)")
    rng = np.random.default_rng(83)
    n, nf = 3000, 200
    xs = rng.uniform(-0.5, 0.5, (n, 3))
    q = rng.standard_normal((n, 3))
    _write_points(tmp_path / "src.txt", np.hstack([xs, q]), 3, "M")
    _write_points(tmp_path / "fld.txt", rng.uniform(-0.5, 0.5, (nf, 3)), 0, "F")
    runs = [subprocess.run([b, "-s", str(tmp_path / "src.txt"), "-f", str(tmp_path / "fld.txt"),
                            *args], capture_output=True, text=True, timeout=300,
                           env=dict(os.environ, MALLOC_MMAP_THRESHOLD_=str(32 << 20)))
            for b in (ref_bin, b200_bin)]
    for r in runs:
        assert r.returncode == 0, r.stderr[-2000:]
    a, b = [_read_fields(r.stdout) for r in runs]
    ncol = 3 + (12 if "-g" in args else 3)
    assert a.shape == b.shape == (nf, ncol)
    assert np.array_equal(a[:, :3], b[:, :3])
    tol = 1e-5 if tool.endswith("-float") else 1e-10
    fa, fb = a[:, 3:6], b[:, 3:6]        # the three potentials, or the curl
    assert np.linalg.norm(fb - fa) <= tol * np.linalg.norm(fa), np.linalg.norm(fb - fa) / np.linalg.norm(fa)
    if ncol > 6:
        # the curl's gradient: the reference's expansion evaluation of it is
        # not the derivative of its curl evaluation (see
        # test_reference_local_curl_gradient_is_inexact), the drop-in's is, so
        # both are held to the reference's direct curl gradient: the drop-in
        # at least as close as the reference's own FMM
        from oracle.oracle_api import Reference
        d = Reference().direct_curl_gradient(np.loadtxt(tmp_path / "src.txt", skiprows=1)[:, :3],
                                             np.loadtxt(tmp_path / "src.txt", skiprows=1)[:, 3:],
                                             a[:, :3])[:, 3:]
        err = [np.linalg.norm(f[:, 6:] - d) / np.linalg.norm(d) for f in (a, b)]
        assert err[1] <= 1.05 * err[0], err


FLOAT_DRIVER_CASES = [
    ("wbfmm-tree-calc-float", ["-b", "-d", "3", "-k", "4", "-R", "8", "-S", "8"]),
    ("wbfmm-tree-calc-float", ["-b", "-d", "3", "-k", "4", "-t", "1e-6"]),
    ("wbfmm-laplace-tree-calc-float", ["-b", "-d", "3", "-R", "8", "-S", "8"]),
    ("wbfmm-laplace-tree-calc-float", ["-b", "-d", "3", "-R", "8", "-S", "8", "-g"]),
    ("wbfmm-laplace-tree-calc-float", ["-b", "-d", "3", "-R", "8", "-S", "8", "-l"]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("tool,args", FLOAT_DRIVER_CASES,
                         ids=lambda x: x if isinstance(x, str) else " ".join(x))
def test_reference_float_driver_on_dropin(gpu_lib, tmp_path, tool, args):
    """The reference's single-precision drivers (its own source through its
    make-source-float step, calling the *_f API) built against the
    reference's single-precision build and against this drop-in, whose *_f
    calls run the engine's FP32 form.  The tree order the Helmholtz driver
    writes (-w: t->ip after the refinements) is identical, since the keys
    are computed in FP32 arithmetic as the reference's build computes them;
    the fields agree with the reference's single- and double-precision
    drivers to the FP32 level (the reference's own FP32 build is 7e-7 from
    its FP64 build on these cases, and both print 6 digits)."""
    bins = {k: os.path.join(ROOT, "oracle", "_ref", tool + suffix)
            for k, suffix in (("ref", "-reference"), ("b200", "-b200"))}
    bins["ref64"] = os.path.join(ROOT, "oracle", "_ref",
                                 tool.replace("-float", "") + "-reference")
    if not all(os.path.exists(b) for b in bins.values()):
        pytest.skip("reference drivers not built (needs the reference sources)")
    rng = np.random.default_rng(82)
    n, nf = 3000, 200
    f32 = lambda a: a.astype(np.float32).astype(np.float64)   # noqa: E731
    xs = f32(rng.uniform(-0.5, 0.5, (n, 3)))
    helm = tool.startswith("wbfmm-tree-calc")
    q = f32(rng.standard_normal((n, 2 if helm else 1)))
    # values that are exact FP32 numbers, written in full so that the float
    # and double drivers read the same points
    _write_points(tmp_path / "src.txt", np.hstack([xs, q]), q.shape[1], "M")
    _write_points(tmp_path / "fld.txt", f32(rng.uniform(-0.5, 0.5, (nf, 3))), 0, "F")
    env = dict(os.environ, MALLOC_MMAP_THRESHOLD_=str(32 << 20))

    def run(b, extra=()):
        r = subprocess.run([b, "-s", str(tmp_path / "src.txt"), "-f", str(tmp_path / "fld.txt"),
                            *args, *extra], capture_output=True, text=True, timeout=300, env=env)
        assert r.returncode == 0, r.stderr[-2000:]
        return r

    out = {k: _read_fields(run(b).stdout) for k, b in bins.items()}
    for k in ("ref", "ref64"):
        assert out[k].shape == out["b200"].shape and out["b200"].shape[0] == nf
    f = {k: v[:, 3:] for k, v in out.items()}
    tol = 2e-6
    assert np.all(np.isfinite(f["b200"]))
    assert np.linalg.norm(f["b200"] - f["ref64"]) <= tol * np.linalg.norm(f["ref64"])
    # the reference's own FP32 build overflows at the high coarse-level
    # orders of the truncation rule (-t): NaN fields, which the drop-in's
    # FP32 form (tables generated in FP64) does not share
    if np.all(np.isfinite(f["ref"])):
        assert np.linalg.norm(f["b200"] - f["ref"]) <= tol * np.linalg.norm(f["ref"])
    else:
        assert "-t" in args
    if helm and "-t" not in args:
        order = [[line.split()[1] for line in run(bins[k], ["-w"]).stderr.splitlines()
                  if len(line.split()) == 5 and line.split()[0].isdigit()]
                 for k in ("ref", "b200")]
        assert len(order[0]) == n and order[0] == order[1]
