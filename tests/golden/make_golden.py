"""Generate the golden fixtures in tests/golden/ from the unmodified reference.

Run where the reference sources are present (oracle/build_oracle.py's
REF_ROOT, or WBFMM_REFERENCE_ROOT):  python tests/golden/make_golden.py
It builds oracle/_ref/libwbfmm_ref.so if needed, runs the reference FMM on
small seeded inputs through oracle/ref_harness.c, and stores inputs and
outputs (potential, gradient, t->ip, box {i,n} per level) as .npz files.
The FP64 direct sums (self-excluding) of the CPU restatement are stored
beside them as the accuracy oracle.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.build_oracle import build_reference, build_restatement  # noqa: E402
from oracle.oracle_api import HELMHOLTZ, LAPLACE, Reference, Restatement  # noqa: E402
from wbfmm_b200 import workloads as W  # noqa: E402


def cases():
    out = []
    p = W.laplace_cube(2000, 500, depth=3, order=8, seed=11)
    out.append(("laplace_small", p))
    p = W.helmholtz_cube(2000, k=4.0, depth=3, seed=12)
    p.xt = p.xs[:500].copy()
    p.targets_are_sources = True
    out.append(("helmholtz_small", p))
    # mixed monopole + dipole sources on a sphere (potential only in the
    # reference), Helmholtz and Laplace
    p = W.helmholtz_sphere(2000, 500, k=6.0, depth=3, seed=13, hi=12)
    out.append(("helmholtz_dipole_small", p))
    rng = np.random.default_rng(14)
    xs = rng.uniform(-0.5, 0.5, (2000, 3))
    nrm = rng.standard_normal((2000, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    q = rng.standard_normal(2000)
    d = rng.standard_normal(2000)
    xt = rng.uniform(-0.5, 0.5, (500, 3))
    p = W.Problem("laplace_dipole_small", LAPLACE, 3, [0, 8, 8, 8], [0, 8, 8, 8],
                  0.0, xs, q, xt, normals=nrm, dipoles=d)
    p.x0, p.D = W.fit_box(xs, xt)
    out.append(("laplace_dipole_small", p))
    return out


def main():
    build_restatement()
    if build_reference() is None:
        raise SystemExit("reference sources not found; cannot generate fixtures")
    R, O = Reference(), Restatement()
    for name, p in cases():
        dip = p.dipoles is not None
        grad = not dip
        r = R.fmm(p.problem, p.depth, p.order_s, p.order_r, p.x0, p.D, p.xs, p.q,
                  p.xt, k=p.k, normals=p.normals, dipoles=p.dipoles, pot=True,
                  grad=grad, want_tree=True)
        dpot, dgrad = O.direct(p.problem, p.xs, p.q, p.xt, k=p.k,
                               normals=p.normals, dipoles=p.dipoles, pot=True,
                               grad=True)
        arrays = dict(
            problem=p.problem, depth=p.depth, order_s=np.array(p.order_s),
            order_r=np.array(p.order_r), k=p.k, x0=p.x0, D=p.D, xs=p.xs,
            q=p.q if p.q is not None else np.zeros(0), xt=p.xt,
            normals=p.normals if p.normals is not None else np.zeros(0),
            dipoles=p.dipoles if p.dipoles is not None else np.zeros(0),
            pot=r["pot"], grad=r["grad"] if grad else np.zeros(0),
            ip=r["ip"], boxes=r["boxes"], direct_pot=dpot, direct_grad=dgrad)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **arrays)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
