"""ctypes bindings to the test oracle (test infrastructure only).

* :class:`Restatement` wraps ``oracle/liboracle.so`` -- our CPU restatement of
  the reference's tree / indexing / direct-sum semantics
  (``oracle/wbfmm_oracle.c``).
* :class:`Reference` wraps ``oracle/_ref/libwbfmm_ref.so`` -- the unmodified
  reference sources driven by ``oracle/ref_harness.c``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs import this module.  The product (``wbfmm_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "liboracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libwbfmm_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)

LAPLACE = 1
HELMHOLTZ = 2


def _ptr(a, t=_dp):
    if a is None:
        return C.cast(None, t)
    return a.ctypes.data_as(t)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _load(path):
    if not os.path.exists(path):
        return None
    return C.CDLL(path)


def level_box_offsets(depth: int) -> list[int]:
    """Start of each level in a levels-concatenated box array."""
    offs, o = [], 0
    for level in range(depth + 1):
        offs.append(o)
        o += 8 ** level
    offs.append(o)
    return offs


class Restatement:
    """Our CPU restatement (bit-exact tree/indexing, FP64 direct sums)."""

    def __init__(self, path: str = RESTATEMENT_SO):
        lib = _load(path)
        if lib is None:
            from oracle.build_oracle import build_restatement
            lib = C.CDLL(build_restatement())
        self.lib = lib
        lib.oracle_morton_encode.restype = C.c_uint64
        lib.oracle_morton_encode.argtypes = [C.c_uint32] * 3
        lib.oracle_point_index_3d.restype = C.c_uint64
        lib.oracle_point_index_3d.argtypes = [_dp, _dp, C.c_double]
        lib.oracle_point_box.restype = C.c_uint64
        lib.oracle_point_box.argtypes = [_dp, C.c_double, C.c_uint, _dp]
        lib.oracle_tree_build.restype = C.c_int
        lib.oracle_tree_build.argtypes = [_dp, C.c_double, C.c_int, C.c_int, _dp,
                                          C.c_int, _up, _up, _ip]
        lib.oracle_box_neighbours.restype = C.c_int
        lib.oracle_box_neighbours.argtypes = [C.c_uint, C.c_uint64, _u64p]
        lib.oracle_interaction_list_4.restype = C.c_int
        lib.oracle_interaction_list_4.argtypes = [C.c_uint, C.c_uint64, _u64p]
        lib.oracle_direct.restype = C.c_int
        lib.oracle_direct.argtypes = [C.c_int, C.c_double, C.c_int, _dp, _dp, _dp,
                                      _dp, C.c_int, _dp, _dp, _dp, C.c_int]

    def point_index_3d(self, x, c, D):
        x = _f64(x); c = _f64(c)
        return int(self.lib.oracle_point_index_3d(_ptr(x), _ptr(c), D))

    def point_box(self, x0, D, level, x):
        x0 = _f64(x0); x = _f64(x)
        return int(self.lib.oracle_point_box(_ptr(x0), D, level, _ptr(x)))

    def tree_build(self, x0, D, depth, pts):
        pts = _f64(pts).reshape(-1, 3)
        n = pts.shape[0]
        x0 = _f64(x0)
        ip = np.zeros(max(n, 1), dtype=np.uint32)
        nbox = level_box_offsets(depth)[-1]
        boxes = np.zeros(2 * nbox, dtype=np.uint32)
        bad = C.c_int(-1)
        rc = self.lib.oracle_tree_build(_ptr(x0), D, depth, n, _ptr(pts), 3,
                                        _ptr(ip, _up), _ptr(boxes, _up), C.byref(bad))
        if rc != 0:
            raise ValueError(f"point {bad.value} not strictly inside the tree cube")
        return ip[:n], boxes.reshape(-1, 2)

    def neighbours(self, level, idx):
        out = np.zeros(27, dtype=np.uint64)
        n = self.lib.oracle_box_neighbours(level, idx, _ptr(out, _u64p))
        return out[:n]

    def interaction_list_4(self, level, idx):
        out = np.zeros(2 * 189, dtype=np.uint64)
        n = self.lib.oracle_interaction_list_4(level, idx, _ptr(out, _u64p))
        return out[: 2 * n].reshape(-1, 2)

    def direct(self, problem, xs, q, xt, k=0.0, normals=None, dipoles=None,
               pot=True, grad=True, nthreads=None):
        xs = _f64(xs).reshape(-1, 3); xt = _f64(xt).reshape(-1, 3)
        q = _f64(q); normals = _f64(normals); dipoles = _f64(dipoles)
        nt = xt.shape[0]
        w = 1 if problem == LAPLACE else 2
        po = np.zeros(nt * w) if pot else None
        go = np.zeros(nt * 3 * w) if grad else None
        if nthreads is None:
            nthreads = os.cpu_count() or 1
        self.lib.oracle_direct(problem, k, xs.shape[0], _ptr(xs), _ptr(q),
                               _ptr(normals), _ptr(dipoles), nt, _ptr(xt),
                               _ptr(po), _ptr(go), nthreads)
        return po, go


class Reference:
    """The unmodified reference (oracle/_ref), driven by ref_harness.c."""

    def __init__(self, path: str = REFERENCE_SO):
        lib = _load(path)
        if lib is None:
            raise FileNotFoundError(path)
        self.lib = lib
        # The reference's dipole P2M touches coefficient index -1 at n = 0
        # (src/expansions.c:363-371, zero weight): 128 bytes before the first
        # box of a level.  Arrays below 32 MiB then come from the heap, where
        # that address is mapped, instead of page-aligned mmap regions.
        try:
            C.CDLL(None).mallopt(-3, 32 << 20)     # M_MMAP_THRESHOLD
        except (AttributeError, OSError):
            pass
        lib.ref_fmm_run.restype = C.c_int
        lib.ref_fmm_run.argtypes = [C.c_int, C.c_int, _ip, _ip, C.c_double, C.c_int,
                                    C.c_int, _dp, C.c_double, C.c_int, _dp, _dp, _dp,
                                    _dp, C.c_int, _dp, _dp, _dp, _up, _up, _dp, _dp,
                                    _dp]
        lib.ref_interaction_list_4.restype = C.c_int
        lib.ref_interaction_list_4.argtypes = [C.c_uint, C.c_uint64, _u64p]
        lib.ref_box_neighbours.restype = C.c_int
        lib.ref_box_neighbours.argtypes = [C.c_uint, C.c_uint64, _u64p]
        lib.ref_point_index_3d.restype = C.c_uint64
        lib.ref_point_index_3d.argtypes = [_dp, _dp, C.c_double]
        lib.ref_point_box.restype = C.c_uint64
        lib.ref_point_box.argtypes = [_dp, C.c_double, C.c_uint, _dp]
        lib.ref_rotation_H.argtypes = [C.c_int, C.c_double, _dp]
        lib.ref_coaxial_SR.argtypes = [C.c_int, C.c_double, _dp]
        lib.ref_coaxial_RR.argtypes = [C.c_int, C.c_double, _dp]
        lib.ref_direct_helmholtz.argtypes = [C.c_double, C.c_int, _dp, _dp, _dp, _dp,
                                             C.c_int, _dp, C.c_int, _dp]
        lib.ref_direct_laplace.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_int, _dp,
                                           C.c_int, _dp]
        lib.wbfmm_laplace_field_direct.restype = C.c_int
        lib.wbfmm_laplace_field_direct.argtypes = [_dp, C.c_int, _dp, C.c_int, C.c_int, _dp,
                                                   C.c_int, _dp, C.c_int, C.c_int, C.c_uint,
                                                   _dp, _dp, C.c_int]

    def fmm(self, problem, depth, order_s, order_r, x0, D, xs, q, xt, k=0.0,
            normals=None, dipoles=None, pot=True, grad=True, bw=False,
            nthreads=1, want_tree=False, want_coeffs=False):
        """Run the reference FMM; returns a dict of outputs and phase times."""
        xs = _f64(xs).reshape(-1, 3); xt = _f64(xt).reshape(-1, 3)
        q = _f64(q); normals = _f64(normals); dipoles = _f64(dipoles)
        ns, nt = xs.shape[0], xt.shape[0]
        os_ = np.zeros(17, dtype=np.int32); or_ = np.zeros(17, dtype=np.int32)
        for lv in range(1, depth + 1):
            os_[lv] = order_s[lv]; or_[lv] = order_r[lv]
        w = 2 if problem == HELMHOLTZ else 1
        po = np.zeros(nt * w) if pot else None
        go = np.zeros(nt * 3 * w) if grad else None
        ip = np.zeros(ns, dtype=np.uint32) if want_tree else None
        boxes = (np.zeros(2 * level_box_offsets(depth)[-1], dtype=np.uint32)
                 if want_tree else None)
        mps = mpr = None
        if want_coeffs:
            ncs = sum(8 ** lv * (order_s[lv] + 1) ** 2 * w for lv in range(1, depth + 1))
            ncr = sum(8 ** lv * (order_r[lv] + 1) ** 2 * w for lv in range(1, depth + 1))
            mps = np.zeros(ncs); mpr = np.zeros(ncr)
        times = np.zeros(6)
        x0 = _f64(x0)
        self.lib.ref_fmm_run(problem, depth, _ptr(os_, _ip), _ptr(or_, _ip), k,
                             int(bw), nthreads, _ptr(x0), D, ns, _ptr(xs), _ptr(q),
                             _ptr(normals), _ptr(dipoles), nt, _ptr(xt), _ptr(po),
                             _ptr(go), _ptr(ip, _up), _ptr(boxes, _up), _ptr(mps),
                             _ptr(mpr), _ptr(times))
        out = {"pot": po, "grad": go, "times": times}
        if want_tree:
            out["ip"] = ip
            out["boxes"] = boxes.reshape(-1, 2)
        if want_coeffs:
            out["mps"] = mps; out["mpr"] = mpr
        return out

    def interaction_list_4(self, level, idx):
        out = np.zeros(2 * 189, dtype=np.uint64)
        n = self.lib.ref_interaction_list_4(level, idx, _ptr(out, _u64p))
        return out[: 2 * n].reshape(-1, 2)

    def neighbours(self, level, idx):
        out = np.zeros(27, dtype=np.uint64)
        n = self.lib.ref_box_neighbours(level, idx, _ptr(out, _u64p))
        return out[:n]

    def point_index_3d(self, x, c, D):
        x = _f64(x); c = _f64(c)
        return int(self.lib.ref_point_index_3d(_ptr(x), _ptr(c), D))

    def point_box(self, x0, D, level, x):
        x0 = _f64(x0); x = _f64(x)
        return int(self.lib.ref_point_box(_ptr(x0), D, level, _ptr(x)))

    def rotation_H(self, N, th):
        n = N + 1
        nerot = (n * (4 * n + 3) * (n + 1)) // 6 + (2 * n) * (n + 1) + n  # generous
        H = np.zeros(nerot + 64)
        self.lib.ref_rotation_H(N, th, _ptr(H))
        return H

    def coaxial_SR(self, L, kr):
        ne = (L + 1) * (L + 2) * (L + 3) // 6 + (L + 1) * (L + 2) // 2 + L + 1
        c = np.zeros(2 * ne)
        self.lib.ref_coaxial_SR(L, kr, _ptr(c))
        return c

    def coaxial_RR(self, L, kr):
        ne = (L + 1) * (L + 2) * (L + 3) // 6 + (L + 1) * (L + 2) // 2 + L + 1
        c = np.zeros(ne)
        self.lib.ref_coaxial_RR(L, kr, _ptr(c))
        return c

    def direct(self, problem, xs, q, xt, k=0.0, normals=None, dipoles=None,
               grad=False):
        xs = _f64(xs).reshape(-1, 3); xt = _f64(xt).reshape(-1, 3)
        q = _f64(q); normals = _f64(normals); dipoles = _f64(dipoles)
        nt = xt.shape[0]
        if problem == HELMHOLTZ:
            f = np.zeros(nt * (6 if grad else 2))
            self.lib.ref_direct_helmholtz(k, xs.shape[0], _ptr(xs), _ptr(q),
                                          _ptr(normals), _ptr(dipoles), nt,
                                          _ptr(xt), int(grad), _ptr(f))
        else:
            f = np.zeros(nt * (3 if grad else 1))
            self.lib.ref_direct_laplace(xs.shape[0], _ptr(xs), _ptr(q),
                                        _ptr(normals), _ptr(dipoles), nt,
                                        _ptr(xt), int(grad), _ptr(f))
        return f


    def direct_curl(self, xs, q3, xt):
        """The reference's direct Laplace curl (WBFMM_FIELD_CURL, nq = 3,
        src/direct-laplace.c:87-130, 274-340), one target at a time."""
        xs = _f64(xs).reshape(-1, 3); q3 = _f64(q3).reshape(-1, 3)
        xt = _f64(xt).reshape(-1, 3)
        out = np.zeros((xt.shape[0], 3))
        for j in range(xt.shape[0]):
            xf = np.ascontiguousarray(xt[j]); f = np.zeros(3)
            self.lib.wbfmm_laplace_field_direct(_ptr(xs), 3, None, 0, xs.shape[0], _ptr(q3), 3,
                                                None, 0, 3, 4, _ptr(xf), _ptr(f), 3)
            out[j] = f
        return out


    def direct_curl_gradient(self, xs, q3, xt):
        """The reference's direct Laplace curl and curl gradient
        (WBFMM_FIELD_CURL | WBFMM_FIELD_GRADIENT, nq = 3,
        src/direct-laplace.c:132-198, 274-340): [nt, 12], the curl then
        d/dx, d/dy, d/dz of its three components, one target at a time."""
        xs = _f64(xs).reshape(-1, 3); q3 = _f64(q3).reshape(-1, 3)
        xt = _f64(xt).reshape(-1, 3)
        out = np.zeros((xt.shape[0], 12))
        for j in range(xt.shape[0]):
            xf = np.ascontiguousarray(xt[j]); f = np.zeros(12)
            self.lib.wbfmm_laplace_field_direct(_ptr(xs), 3, None, 0, xs.shape[0], _ptr(q3), 3,
                                                None, 0, 3, 4 | 2, _ptr(xf), _ptr(f), 12)
            out[j] = f
        return out


def curl_from_gradients(g):
    """curl_i = e_ijk d_j A_k from the gradients g[k] ([nt, 3]) of the three
    components of a vector potential."""
    gx, gy, gz = (np.asarray(a).reshape(-1, 3) for a in g)
    return np.stack([gz[:, 1] - gy[:, 2], gx[:, 2] - gz[:, 0], gy[:, 0] - gx[:, 1]], axis=1)


def have_reference() -> bool:
    return os.path.exists(REFERENCE_SO)
