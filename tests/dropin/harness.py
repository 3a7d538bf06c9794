"""Build and run tests/dropin/driver.c, a wbfmm.h client program, against
either library:

* ``b200``: include/wbfmm.h + wbfmm_b200/libwbfmm_b200.so (the product);
* ``reference``: the reference's own header and the test oracle's build of
  the unmodified reference sources (oracle/_ref/libwbfmm_ref.so).  Built only
  where the reference tree is present; the binary is kept in
  tests/dropin/_build so later runs can use it without the sources.

Test infrastructure only.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BUILD = os.path.join(HERE, "_build")
SRC = os.path.join(HERE, "driver.c")
sys.path.insert(0, ROOT)
from oracle.build_oracle import REF_ROOT  # noqa: E402  (the reference tree, if present)

LAPLACE, HELMHOLTZ = 1, 2
POTENTIAL, GRADIENT = 1, 2


@dataclass
class Case:
    problem: int
    depth: int
    order_s: list
    order_r: list
    k: float
    x0: np.ndarray
    D: float
    xs: np.ndarray
    xt: np.ndarray
    q: np.ndarray | None = None
    normals: np.ndarray | None = None
    dipoles: np.ndarray | None = None
    mode: int = 0          # 0: target by target, 1: target list
    field: int = POTENTIAL
    bw: int = 0

    @property
    def w(self):
        return 2 if self.problem == HELMHOLTZ else 1


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def driver_path(kind: str) -> str:
    return os.path.join(BUILD, f"driver_{kind}")


def build_driver(kind: str) -> str | None:
    """Compile the driver for `kind`; None when it cannot be built here."""
    os.makedirs(BUILD, exist_ok=True)
    out = driver_path(kind)
    if kind == "b200":
        lib_dir = os.path.join(ROOT, "wbfmm_b200")
        lib = os.path.join(lib_dir, "libwbfmm_b200.so")
        deps = [SRC, os.path.join(ROOT, "include", "wbfmm.h"), lib]
        if _newer(out, deps):
            subprocess.run(["gcc", "-O2", "-std=c11", "-Wall", "-Werror",
                            "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
                            lib, f"-Wl,-rpath,{lib_dir}", "-lm"], check=True)
        return out
    if kind == "reference":
        lib_dir = os.path.join(ROOT, "oracle", "_ref")
        lib = os.path.join(lib_dir, "libwbfmm_ref.so")
        hdr = os.path.join(REF_ROOT, "src", "wbfmm.h")
        if not os.path.exists(lib):
            return None
        if not os.path.exists(hdr):
            return out if os.path.exists(out) else None
        if _newer(out, [SRC, hdr, lib]):
            subprocess.run(["gcc", "-O2", "-I", os.path.join(ROOT, "oracle", "shim"),
                            "-I", os.path.join(REF_ROOT, "src"), "-I", REF_ROOT,
                            SRC, "-o", out, lib, f"-Wl,-rpath,{lib_dir}",
                            "-lm", "-fopenmp", "-pthread"], check=True)
        return out
    raise ValueError(kind)


def write_input(c: Case, path: str) -> None:
    ns, nt = len(c.xs), len(c.xt)
    hdr = np.array([c.problem, c.depth, ns, nt, c.q is not None,
                    c.normals is not None, c.dipoles is not None, c.mode,
                    c.field, c.bw], dtype=np.int32)
    with open(path, "wb") as f:
        hdr.tofile(f)
        np.array([c.k, *c.x0, c.D], dtype=np.float64).tofile(f)
        np.asarray(c.order_s, dtype=np.int32).tofile(f)
        np.asarray(c.order_r, dtype=np.int32).tofile(f)
        np.ascontiguousarray(c.xs, dtype=np.float64).tofile(f)
        for a in (c.q, c.normals, c.dipoles):
            if a is not None:
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        np.ascontiguousarray(c.xt, dtype=np.float64).tofile(f)


def read_output(c: Case, path: str) -> dict:
    raw = open(path, "rb").read()
    ns, nt, w = len(c.xs), len(c.xt), c.w
    nf = 3 * w if c.field & GRADIENT else w
    off = 0

    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=n, offset=off)
        off += a.nbytes
        return a.copy()

    out = {"f": take(np.float64, nt * nf).reshape(nt, nf),
           "ip": take(np.uint32, ns)}
    for level in range(c.depth + 1):
        out[f"boxes{level}"] = take(np.uint32, 2 * 8 ** level).reshape(-1, 2)
    for level in range(1, c.depth + 1):
        out[f"mps{level}"] = take(np.float64, 8 ** level * (c.order_s[level] + 1) ** 2 * w)
        out[f"mpr{level}"] = take(np.float64, 8 ** level * (c.order_r[level] + 1) ** 2 * w)
    assert off == len(raw), "driver output size mismatch"
    return out


def run(kind: str, c: Case, timeout: float = 600) -> dict:
    exe = build_driver(kind)
    if exe is None:
        raise FileNotFoundError(f"driver for {kind} cannot be built here")
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        write_input(c, fi)
        env = dict(os.environ)
        if kind == "reference":
            # The reference's dipole P2M touches coefficient index -1 at
            # n = 0 (src/expansions.c:363-371, zero weight).  For the
            # first box of a level that is 128 bytes before the array; an
            # mmap'd array then faults when the page before it is unmapped.
            # Serving coefficient arrays from the heap keeps that read in
            # mapped memory.
            env["MALLOC_MMAP_THRESHOLD_"] = str(32 << 20)
        r = subprocess.run([exe, fi, fo], capture_output=True, text=True,
                           timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"driver_{kind} exited {r.returncode}: {r.stderr[-2000:]}")
        return read_output(c, fo)


def cases() -> dict:
    """Small seeded client workloads: both problems, both evaluation modes,
    monopoles and mixed monopole + dipole sources."""
    out = {}

    def box(xs, xt):
        lo = np.minimum(xs.min(0), xt.min(0)) - 0.01
        D = float((np.maximum(xs.max(0), xt.max(0)) - lo).max() + 0.02)
        return lo, D

    rng = np.random.default_rng(41)
    xs = rng.uniform(-1, 1, (1500, 3))
    xt = rng.uniform(-1, 1, (200, 3))
    x0, D = box(xs, xt)
    q = rng.standard_normal((1500, 2))
    out["helm_point_pot"] = Case(HELMHOLTZ, 3, [0, 8, 8, 7], [0, 8, 8, 7], 3.0,
                                 x0, D, xs, xt, q=q)
    nrm = rng.standard_normal((1500, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    dip = rng.standard_normal((1500, 2))
    # the reference's near-field gradient takes monopoles only
    # (src/local.c:234-262, src/local-laplace.c:1136-1163)
    out["helm_point_pot_dipole"] = Case(HELMHOLTZ, 3, [0, 8, 8, 7], [0, 8, 8, 7],
                                        3.0, x0, D, xs, xt, q=q, normals=nrm,
                                        dipoles=dip)
    out["helm_point_grad"] = Case(HELMHOLTZ, 3, [0, 8, 8, 7], [0, 8, 8, 7], 3.0,
                                  x0, D, xs, xt, q=q, field=GRADIENT)
    out["helm_list_pot"] = Case(HELMHOLTZ, 3, [0, 8, 8, 7], [0, 8, 8, 7], 3.0,
                                x0, D, xs, xt, q=q, mode=1)
    ql = rng.standard_normal(1500)
    dl = rng.standard_normal(1500)
    out["lap_point_grad"] = Case(LAPLACE, 3, [0, 8, 8, 8], [0, 8, 8, 8], 0.0,
                                 x0, D, xs, xt, q=ql, field=GRADIENT)
    out["lap_point_pot_dipole"] = Case(LAPLACE, 3, [0, 8, 8, 8], [0, 8, 8, 8],
                                       0.0, x0, D, xs, xt, q=ql, normals=nrm,
                                       dipoles=dl)
    out["lap_list_pot_dipole"] = Case(LAPLACE, 3, [0, 8, 8, 8], [0, 8, 8, 8],
                                      0.0, x0, D, xs, xt, q=ql, normals=nrm,
                                      dipoles=dl, mode=1)
    return out
