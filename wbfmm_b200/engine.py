"""Python host binding of the engine's C ABI (include/wbfmm_b200.h).

The binding loads ``libwbfmm_b200.so`` from this package directory and fails
loudly if it is missing: there is no CPU fallback.  Arrays are NumPy FP64 on
the host, or anything exposing a device pointer (``torch`` CUDA tensors,
``int`` addresses) with ``on_device=True``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwbfmm_b200.so")

LAPLACE = 1
HELMHOLTZ = 2
FP64 = 0
FP32 = 1
POTENTIAL = 1
GRADIENT = 2
MAX_DEPTH = 16

STATUS = {
    0: "ok", -1: "invalid argument", -2: "point outside the tree cube",
    -3: "expansion order unsupported", -4: "call out of sequence",
    -5: "device allocation failed", -6: "over the device-memory budget",
    -7: "no CUDA device",
}


class WbfmmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"wbfmm_b200 error {code} ({STATUS.get(code, 'CUDA')}): {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("problem", C.c_int), ("depth", C.c_int),
        ("order_s", C.c_int * (MAX_DEPTH + 1)),
        ("order_r", C.c_int * (MAX_DEPTH + 1)),
        ("k", C.c_double), ("x0", C.c_double * 3), ("D", C.c_double),
        ("precision", C.c_int), ("field", C.c_int), ("skip_empty", C.c_int),
        ("managed", C.c_int), ("leaf_order", C.c_int), ("keys_fp32", C.c_int),
        ("near_fp32", C.c_int), ("sparse", C.c_int),
    ]


class Request(C.Structure):
    _fields_ = [
        ("cfg", Config), ("nsrc", C.c_int), ("xs", C.c_void_p),
        ("q", C.c_void_p), ("normals", C.c_void_p), ("dipoles", C.c_void_p),
        ("ntgt", C.c_int), ("xt", C.c_void_p), ("pot", C.c_void_p),
        ("grad", C.c_void_p), ("arrival", C.c_double), ("on_device", C.c_int),
    ]


_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libwbfmm_b200.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m wbfmm_b200.build` "
            "(the library has no CPU fallback)")
    lib = C.CDLL(path)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
    u32p = C.POINTER(C.c_uint32)
    sigs = {
        "wbfmm_b200_last_error": (C.c_char_p, []),
        "wbfmm_b200_device_count": (ip, []),
        "wbfmm_b200_solver_create": (ip, [C.POINTER(vp), C.POINTER(Config), vp]),
        "wbfmm_b200_solver_destroy": (ip, [vp]),
        "wbfmm_b200_footprint": (C.c_int64, [C.POINTER(Config), C.c_int64, C.c_int64]),
        "wbfmm_b200_set_sources": (ip, [vp, ip, vp, ip, vp, ip, ip]),
        "wbfmm_b200_set_strengths": (ip, [vp, vp, ip, vp, ip, ip]),
        "wbfmm_b200_set_targets": (ip, [vp, ip, vp, ip, ip]),
        "wbfmm_b200_build_operators": (ip, [vp]),
        "wbfmm_b200_leaf_expansions": (ip, [vp]),
        "wbfmm_b200_upward_pass": (ip, [vp, ip]),
        "wbfmm_b200_downward_pass": (ip, [vp, ip]),
        "wbfmm_b200_evaluate": (ip, [vp]),
        "wbfmm_b200_run": (ip, [vp]),
        "wbfmm_b200_run_async": (ip, [vp]),
        "wbfmm_b200_run_graph": (ip, [vp]),
        "wbfmm_b200_wait": (ip, [vp]),
        "wbfmm_b200_set_deferred_checks": (ip, [vp, ip]),
        "wbfmm_b200_selftest_sincos": (ip, [C.c_double, ip, dp]),
        "wbfmm_b200_fp32_fma_peak": (ip, [dp]),
        "wbfmm_b200_error_norms": (ip, [C.c_int64, vp, vp, ip, dp]),
        "wbfmm_b200_laplace_curl": (ip, [vp, vp, ip, vp, ip]),
        "wbfmm_b200_laplace_curl_gradient": (ip, [vp, vp, ip, vp, ip]),
        "wbfmm_b200_laplace_hessian": (ip, [vp, vp, ip, ip]),
        "wbfmm_b200_target_bases": (ip, [vp]),
        "wbfmm_b200_set_evaluation": (ip, [vp, ip, ip]),
        "wbfmm_b200_evaluate_bases": (ip, [vp, ip]),
        "wbfmm_b200_synchronize": (ip, [vp]),
        "wbfmm_b200_get_field": (ip, [vp, vp, vp, ip]),
        "wbfmm_b200_get_tree": (ip, [vp, u32p, u32p, u32p, ip]),
        "wbfmm_b200_get_coefficients": (ip, [vp, ip, dp, dp]),
        "wbfmm_b200_coefficient_pointers": (ip, [vp, ip, C.POINTER(vp), C.POINTER(vp)]),
        "wbfmm_b200_coefficient_storage": (ip, [vp, ip, C.POINTER(C.c_int64),
                                                C.POINTER(C.c_int64)]),
        "wbfmm_b200_stage_times": (ip, [vp, dp]),
        "wbfmm_b200_kernel_launches": (C.c_int64, [vp]),
        "wbfmm_b200_solve": (ip, [C.POINTER(Config), ip, vp, vp, vp, vp, ip, vp, vp, vp]),
        "wbfmm_b200_invalidate_operators": (ip, [vp]),
        "wbfmm_b200_m2l": (ip, [vp, ip]),
        "wbfmm_b200_set_m2l_kernel": (ip, [vp, ip]),
        "wbfmm_b200_l2l": (ip, [vp, ip]),
        "wbfmm_b200_direct": (ip, [ip, C.c_double, ip, vp, vp, vp, vp, ip, vp, vp, vp, ip]),
        "wbfmm_b200_fp32_range_ok": (ip, [C.POINTER(Config)]),
        "wbfmm_b200_server_create": (ip, [C.POINTER(vp), ip, C.c_int64]),
        "wbfmm_b200_server_destroy": (ip, [vp]),
        "wbfmm_b200_server_clock": (C.c_double, [vp]),
        "wbfmm_b200_server_submit": (ip, [vp, C.POINTER(Request), C.POINTER(C.c_int64)]),
        "wbfmm_b200_server_poll": (ip, [vp, C.c_int64]),
        "wbfmm_b200_server_set_order": (ip, [vp, ip]),
        "wbfmm_b200_server_wait": (ip, [vp, C.c_int64]),
        "wbfmm_b200_server_times": (ip, [vp, C.c_int64, dp]),
        "wbfmm_b200_server_forget": (ip, [vp, C.c_int64]),
        "wbfmm_b200_server_drain": (ip, [vp]),
        "wbfmm_b200_server_stats": (ip, [vp, C.POINTER(C.c_int64)]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        msg = load_library().wbfmm_b200_last_error().decode(errors="replace")
        raise WbfmmError(rc, msg)


def _addr(a):
    """Address of a host array / device tensor / raw int pointer (or None)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)}")


def _host(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class SolverConfig:
    problem: int
    depth: int
    order_s: list
    order_r: list
    k: float = 0.0
    x0: tuple = (0.0, 0.0, 0.0)
    D: float = 1.0
    precision: int = FP64
    field: int = POTENTIAL | GRADIENT
    skip_empty: bool = False
    managed: bool = False
    leaf_order: bool = False
    near_fp32: bool = False
    sparse: bool = False

    def to_c(self) -> Config:
        c = Config()
        c.problem = self.problem
        c.depth = self.depth
        for lv in range(MAX_DEPTH + 1):
            c.order_s[lv] = int(self.order_s[lv]) if lv < len(self.order_s) else 0
            c.order_r[lv] = int(self.order_r[lv]) if lv < len(self.order_r) else 0
        c.k = float(self.k)
        for i in range(3):
            c.x0[i] = float(self.x0[i])
        c.D = float(self.D)
        c.precision = self.precision
        c.field = self.field
        c.skip_empty = int(bool(self.skip_empty))
        c.managed = int(bool(self.managed))
        c.leaf_order = int(bool(self.leaf_order))
        c.near_fp32 = int(bool(self.near_fp32))
        c.sparse = int(bool(self.sparse))
        return c

    @staticmethod
    def from_problem(p, precision=FP64, field=POTENTIAL | GRADIENT,
                     skip_empty=False, leaf_order=False, near_fp32=False,
                     sparse=False) -> "SolverConfig":
        return SolverConfig(p.problem, p.depth, list(p.order_s), list(p.order_r),
                            p.k, tuple(p.x0), p.D, precision, field, skip_empty,
                            False, leaf_order, near_fp32, sparse)


class Solver:
    """One FMM solve on the GPU (see include/wbfmm_b200.h)."""

    def __init__(self, cfg: SolverConfig, stream: int | None = None):
        self.lib = load_library()
        self.cfg = cfg
        self._c = cfg.to_c()
        h = C.c_void_p()
        _check(self.lib.wbfmm_b200_solver_create(C.byref(h), C.byref(self._c), stream))
        self.h = h
        self.ns = self.nt = 0
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.wbfmm_b200_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_sources(self, xs, normals=None, on_device=False, xstr=3, nstr=3):
        if not on_device:
            xs = _host(xs).reshape(-1, 3)
            normals = _host(normals)
            n = xs.shape[0]
        else:
            n = int(xs.shape[0]) if hasattr(xs, "shape") else None
        self._keep = [xs, normals]
        _check(self.lib.wbfmm_b200_set_sources(self.h, n, _addr(xs), xstr,
                                               _addr(normals), nstr, int(on_device)))
        self.ns = n
        return self

    def set_strengths(self, q=None, dipoles=None, on_device=False):
        w = 2 if self.cfg.problem == HELMHOLTZ else 1
        if not on_device:
            q = _host(q); dipoles = _host(dipoles)
        _check(self.lib.wbfmm_b200_set_strengths(self.h, _addr(q), w, _addr(dipoles),
                                                 w, int(on_device)))
        return self

    def set_targets(self, xt, on_device=False, tstr=3):
        if not on_device:
            xt = _host(xt).reshape(-1, 3)
        n = int(xt.shape[0])
        _check(self.lib.wbfmm_b200_set_targets(self.h, n, _addr(xt), tstr, int(on_device)))
        self.nt = n
        return self

    def build_operators(self):
        _check(self.lib.wbfmm_b200_build_operators(self.h))

    def leaf_expansions(self):
        _check(self.lib.wbfmm_b200_leaf_expansions(self.h))

    def upward_pass(self, level):
        _check(self.lib.wbfmm_b200_upward_pass(self.h, level))

    def downward_pass(self, level):
        _check(self.lib.wbfmm_b200_downward_pass(self.h, level))

    def set_m2l_kernel(self, mode):
        """0 warp per target, 1 automatic (default), 2 lane per pair, 3 target
        tiles; True / False select 1 / 0."""
        _check(self.lib.wbfmm_b200_set_m2l_kernel(self.h, int(mode)))

    def m2l(self, level):
        _check(self.lib.wbfmm_b200_m2l(self.h, level))

    def l2l(self, level):
        _check(self.lib.wbfmm_b200_l2l(self.h, level))

    def evaluate(self):
        _check(self.lib.wbfmm_b200_evaluate(self.h))

    def run(self):
        _check(self.lib.wbfmm_b200_run(self.h))
        return self

    def run_async(self):
        """Queue every pass on the solver's stream; wait() blocks."""
        _check(self.lib.wbfmm_b200_run_async(self.h))
        return self

    def laplace_curl(self, q3):
        """Curl of the vector potential of sources with 3-vector strengths
        q3 [ns, 3] at the targets: [nt, 3] (Laplace solver, gradient field)."""
        q3 = _host(q3).reshape(-1, 3)
        out = np.zeros(self.nt * 3)
        _check(self.lib.wbfmm_b200_laplace_curl(self.h, _addr(q3), 3, _addr(out), 0))
        return out.reshape(-1, 3)

    def laplace_curl_gradient(self, q3):
        """Curl of the vector potential of sources with 3-vector strengths
        q3 [ns, 3] and its gradient at the targets: [nt, 12] (curl, then
        d/dx, d/dy, d/dz of the curl; Laplace solver, gradient field)."""
        q3 = _host(q3).reshape(-1, 3)
        out = np.zeros(self.nt * 12)
        _check(self.lib.wbfmm_b200_laplace_curl_gradient(self.h, _addr(q3), 3, _addr(out), 0))
        return out.reshape(-1, 12)

    def hessian(self, neighbours=True):
        """Second derivatives of the potential at the targets after run():
        [nt, 3, 3] (Laplace solver)."""
        out = np.zeros(self.nt * 9)
        _check(self.lib.wbfmm_b200_laplace_hessian(self.h, _addr(out), int(bool(neighbours)), 0))
        return out.reshape(-1, 3, 3)

    def set_evaluation(self, field, neighbours=True):
        """Fields written by evaluate() (a subset of the configured ones) and
        whether the near field (P2P) is added."""
        _check(self.lib.wbfmm_b200_set_evaluation(self.h, int(field), int(bool(neighbours))))
        return self

    def target_bases(self):
        """Precompute the targets' expansion bases and near-field weights
        (potential; kept until the sources or targets change)."""
        _check(self.lib.wbfmm_b200_target_bases(self.h))
        return self

    def evaluate_bases(self, neighbours=True):
        """The potential at the targets from the precomputed bases, the leaf
        expansions of the last downward pass and the current strengths
        (read it with field())."""
        _check(self.lib.wbfmm_b200_evaluate_bases(self.h, int(bool(neighbours))))
        return self

    def run_graph(self):
        """The passes as one CUDA graph launch (captured on the first call
        after a change of tree, targets, tables or options); wait() blocks."""
        _check(self.lib.wbfmm_b200_run_graph(self.h))
        return self

    def wait(self):
        _check(self.lib.wbfmm_b200_wait(self.h))
        return self

    def set_deferred_checks(self, on=True):
        """Domain checks of set_sources / set_targets reported by run / wait
        instead of by the set calls (no host wait inside a solve)."""
        _check(self.lib.wbfmm_b200_set_deferred_checks(self.h, int(bool(on))))
        return self

    def synchronize(self):
        _check(self.lib.wbfmm_b200_synchronize(self.h))

    def field(self):
        w = 2 if self.cfg.problem == HELMHOLTZ else 1
        pot = np.zeros(self.nt * w) if self.cfg.field & POTENTIAL else None
        grad = np.zeros(self.nt * 3 * w) if self.cfg.field & GRADIENT else None
        _check(self.lib.wbfmm_b200_get_field(self.h, _addr(pot), _addr(grad), 0))
        return pot, grad

    def field_to_device(self, pot_ptr=None, grad_ptr=None):
        _check(self.lib.wbfmm_b200_get_field(self.h, pot_ptr, grad_ptr, 1))

    def tree(self, level):
        nb = 8 ** level
        ip = np.zeros(self.ns, dtype=np.uint32)
        bi = np.zeros(nb, dtype=np.uint32)
        bn = np.zeros(nb, dtype=np.uint32)
        u32p = C.POINTER(C.c_uint32)
        _check(self.lib.wbfmm_b200_get_tree(self.h, ip.ctypes.data_as(u32p),
                                            bi.ctypes.data_as(u32p),
                                            bn.ctypes.data_as(u32p), level))
        return ip, bi, bn

    def coefficients(self, level):
        w = 2 if self.cfg.problem == HELMHOLTZ else 1
        nb = 8 ** level
        ms = np.zeros(nb * (self.cfg.order_s[level] + 1) ** 2 * w)
        mr = np.zeros(nb * (self.cfg.order_r[level] + 1) ** 2 * w)
        dp = C.POINTER(C.c_double)
        _check(self.lib.wbfmm_b200_get_coefficients(self.h, level, ms.ctypes.data_as(dp),
                                                    mr.ctypes.data_as(dp)))
        return ms, mr

    def coefficient_storage(self, level=0):
        """(stored groups of eight boxes, device bytes of the coefficient
        arrays) of a level, or totals over all levels for level 0."""
        g, b = C.c_int64(), C.c_int64()
        _check(self.lib.wbfmm_b200_coefficient_storage(self.h, level, C.byref(g), C.byref(b)))
        return g.value, b.value

    def invalidate_operators(self):
        _check(self.lib.wbfmm_b200_invalidate_operators(self.h))

    def stage_times(self):
        t = np.zeros(6)
        _check(self.lib.wbfmm_b200_stage_times(self.h, t.ctypes.data_as(C.POINTER(C.c_double))))
        return dict(zip(["tree", "operators", "p2m", "upward", "downward", "evaluate"], t))

    def kernel_launches(self) -> int:
        return int(self.lib.wbfmm_b200_kernel_launches(self.h))


def solve(p, precision=FP64, field=POTENTIAL | GRADIENT, skip_empty=False, sparse=False):
    """Run one FMM solve of a :class:`wbfmm_b200.workloads.Problem`
    (sparse: sparse level storage)."""
    cfg = SolverConfig.from_problem(p, precision, field, skip_empty, sparse=sparse)
    with Solver(cfg) as s:
        s.set_sources(p.xs, p.normals)
        s.set_strengths(p.q, p.dipoles)
        s.set_targets(p.xt)
        s.run()
        return s.field()


def direct(problem, xs, q, xt, k=0.0, normals=None, dipoles=None, pot=True,
           grad=True):
    """FP64 direct sum on the GPU (self-excluding), host arrays."""
    lib = load_library()
    xs = _host(xs).reshape(-1, 3); xt = _host(xt).reshape(-1, 3)
    q = _host(q); normals = _host(normals); dipoles = _host(dipoles)
    w = 2 if problem == HELMHOLTZ else 1
    po = np.zeros(xt.shape[0] * w) if pot else None
    go = np.zeros(xt.shape[0] * 3 * w) if grad else None
    _check(lib.wbfmm_b200_direct(problem, float(k), xs.shape[0], _addr(xs), _addr(q),
                                 _addr(normals), _addr(dipoles), xt.shape[0], _addr(xt),
                                 _addr(po), _addr(go), 0))
    return po, go


def error_norms(f, ref):
    """GPU FP64 reduction: (||f - ref||_2 / ||ref||_2, max|f - ref| / max|ref|)
    for host arrays of equal size."""
    f = _host(f).ravel(); ref = _host(ref).ravel()
    if f.shape != ref.shape:
        raise ValueError("f and ref differ in size")
    out = (C.c_double * 4)()
    _check(load_library().wbfmm_b200_error_norms(f.size, _addr(f), _addr(ref), 0, out))
    return out[0] / out[1], out[2] / out[3]


def selftest_sincos(xmax: float, n: int):
    """(engine's FP32 near-field sin/cos, CUDA sincosf): largest absolute
    errors against FP64 at n+1 FP32 arguments in [0, xmax]."""
    err = (C.c_double * 2)()
    _check(load_library().wbfmm_b200_selftest_sincos(float(xmax), int(n), err))
    return float(err[0]), float(err[1])


def fp32_fma_peak() -> float:
    """Measured FP32 FMA throughput of the current GPU, TFLOP/s."""
    t = C.c_double()
    _check(load_library().wbfmm_b200_fp32_fma_peak(C.byref(t)))
    return float(t.value)


def device_count() -> int:
    return int(load_library().wbfmm_b200_device_count())


def fp32_range_ok(cfg: "SolverConfig") -> bool:
    """Whether the FP32 form keeps this configuration inside the FP32 range."""
    c = cfg.to_c()
    return bool(load_library().wbfmm_b200_fp32_range_ok(C.byref(c)))


def footprint(cfg: "SolverConfig", ns: int, nt: int) -> int:
    """Device bytes a solve of this configuration holds (admission estimate)."""
    c = cfg.to_c()
    return int(load_library().wbfmm_b200_footprint(C.byref(c), int(ns), int(nt)))


class Server:
    """Served form: continuous batching of independent solves on one GPU
    (wbfmm_b200_server_* in include/wbfmm_b200.h).

    ``submit`` takes a :class:`wbfmm_b200.workloads.Problem` and a precision
    and returns a ticket; the host arrays of a request are held here until
    the request completes, and its fields land in arrays this object owns.
    """

    def __init__(self, slots: int = 16, hbm_budget: int = 150 * 10**9,
                 largest_first: bool = False):
        self._lib = load_library()
        self._h = C.c_void_p()
        _check(self._lib.wbfmm_b200_server_create(C.byref(self._h), int(slots), int(hbm_budget)))
        if largest_first:
            _check(self._lib.wbfmm_b200_server_set_order(self._h, 1))
        self._held = {}

    def close(self):
        if self._h:
            self._lib.wbfmm_b200_server_destroy(self._h)
            self._h = C.c_void_p()
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def clock(self) -> float:
        return float(self._lib.wbfmm_b200_server_clock(self._h))

    def submit(self, p, precision=FP32, field=POTENTIAL | GRADIENT,
               arrival: float = 0.0, skip_empty: bool = False,
               leaf_order: bool = False, device: dict | None = None,
               near_fp32: bool = False) -> int:
        """Queue one solve; skip_empty: no local expansions for boxes
        without targets (the fields at the targets are unchanged);
        leaf_order: sources sorted by leaf box only; near_fp32: an FP64
        solve with its near field in FP32.  With ``device`` (a dict
        of device arrays -- objects with ``data_ptr()`` -- under the keys
        xs, q, normals, dipoles, xt, pot, grad, absent or None where unused)
        the request reads and writes those instead of host arrays; the
        caller keeps them alive until the request completes."""
        cfg = SolverConfig.from_problem(p, precision, field, skip_empty, leaf_order, near_fp32)
        w = 2 if p.problem == HELMHOLTZ else 1
        if device is not None:
            d = {k: device.get(k) for k in ("xs", "q", "normals", "dipoles", "xt", "pot", "grad")}
            if d["xt"] is None:
                d["xt"] = d["xs"]
            r = Request(cfg.to_c(), p.ns, _addr(d["xs"]), _addr(d["q"]), _addr(d["normals"]),
                        _addr(d["dipoles"]), p.nt, _addr(d["xt"]),
                        _addr(d["pot"]) if field & POTENTIAL else None,
                        _addr(d["grad"]) if field & GRADIENT else None, float(arrival), 1)
            t = C.c_int64()
            _check(self._lib.wbfmm_b200_server_submit(self._h, C.byref(r), C.byref(t)))
            self._held[t.value] = (d, None, None, None, None, d["pot"], d["grad"])
            return t.value
        xs = _host(p.xs)
        xt = xs if p.targets_are_sources else _host(p.xt)
        q, nrm, dip = _host(p.q), _host(p.normals), _host(p.dipoles)
        nt = xt.shape[0]
        pot = np.zeros(nt * w) if field & POTENTIAL else None
        grad = np.zeros(nt * 3 * w) if field & GRADIENT else None
        r = Request(cfg.to_c(), xs.shape[0], _addr(xs), _addr(q), _addr(nrm),
                    _addr(dip), nt, _addr(xt), _addr(pot), _addr(grad),
                    float(arrival), 0)
        t = C.c_int64()
        _check(self._lib.wbfmm_b200_server_submit(self._h, C.byref(r), C.byref(t)))
        self._held[t.value] = (xs, xt, q, nrm, dip, pot, grad)
        return t.value

    def done(self, ticket: int) -> bool:
        rc = self._lib.wbfmm_b200_server_poll(self._h, ticket)
        if rc < 0:
            _check(rc)
        return rc == 1

    def wait(self, ticket: int):
        """Block until the request completes; return (pot, grad)."""
        _check(self._lib.wbfmm_b200_server_wait(self._h, ticket))
        held = self._held[ticket]
        return held[5], held[6]

    def times(self, ticket: int):
        """(arrival, start, queued, end) on the server clock, seconds: queued
        is when the solve's device work had all been issued."""
        t = np.zeros(4)
        _check(self._lib.wbfmm_b200_server_times(self._h, ticket, t.ctypes.data_as(C.POINTER(C.c_double))))
        return tuple(float(x) for x in t)

    def forget(self, ticket: int):
        _check(self._lib.wbfmm_b200_server_forget(self._h, ticket))
        self._held.pop(ticket, None)

    def drain(self):
        _check(self._lib.wbfmm_b200_server_drain(self._h))

    def stats(self) -> dict:
        a = (C.c_int64 * 7)()
        _check(self._lib.wbfmm_b200_server_stats(self._h, a))
        keys = ("completed", "peak_bytes_in_flight", "peak_solves_in_flight",
                "table_cache_hits", "table_cache_misses", "table_cache_bytes",
                "kernel_launches")
        return dict(zip(keys, (int(x) for x in a)))
