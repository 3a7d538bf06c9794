"""Golden vectors of the reference's own FP64 direct sums.

Run where the reference sources are present (oracle/build_oracle.py's
REF_ROOT, or WBFMM_REFERENCE_ROOT):  python tests/golden/make_direct_golden.py

The unmodified reference (oracle/_ref/libwbfmm_ref.so) evaluates
wbfmm_total_field / wbfmm_total_field_grad (src/direct.c:35-294) and
wbfmm_laplace_field / wbfmm_laplace_field_grad (src/direct-laplace.c:35-85,
200-263) on seeded sources and targets that never coincide (the reference
has no self-exclusion).  Cases, one source set each:

  helm_mono    Helmholtz monopoles, k = 7.3: potential and gradient
  helm_mixed   Helmholtz monopoles + dipoles along unit normals: potential
               (the reference's gradient stops on dipoles)
  lap_mono     Laplace monopoles: potential and gradient
  lap_dipole   Laplace dipoles only: potential
  lap_mixed    Laplace monopoles + dipoles: potential (the reference leaves
               the 1/(4 pi) off the dipole term here, src/direct-laplace.c:
               261-263; kept as it computes it)

Output: tests/golden/direct_sums.npz, keys "<case>_<array>".
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.build_oracle import build_reference  # noqa: E402
from oracle.oracle_api import HELMHOLTZ, LAPLACE, Reference  # noqa: E402

NS, NT = 2000, 300


def inputs(seed, helm, normals):
    rng = np.random.default_rng(seed)
    xs = rng.uniform(-0.5, 0.5, (NS, 3))
    xt = rng.uniform(-0.5, 0.5, (NT, 3))
    w = 2 if helm else 1
    q = rng.standard_normal(NS * w)
    nrm = dip = None
    if normals:
        nrm = rng.standard_normal((NS, 3))
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        dip = rng.standard_normal(NS * w)
    return xs, xt, q, nrm, dip


def main():
    if build_reference() is None:
        raise SystemExit("reference sources not found; cannot generate fixtures")
    R = Reference()
    out = {}
    cases = [("helm_mono", HELMHOLTZ, False, True, True, 201),
             ("helm_mixed", HELMHOLTZ, True, True, False, 202),
             ("lap_mono", LAPLACE, False, True, True, 203),
             ("lap_dipole", LAPLACE, True, False, False, 204),
             ("lap_mixed", LAPLACE, True, True, False, 205)]
    k = 7.3
    for name, problem, normals, mono, grad, seed in cases:
        helm = problem == HELMHOLTZ
        xs, xt, q, nrm, dip = inputs(seed, helm, normals)
        qq = q if mono else None
        pot = R.direct(problem, xs, qq, xt, k=k, normals=nrm, dipoles=dip, grad=False)
        arrays = {"problem": problem, "k": k if helm else 0.0, "xs": xs, "xt": xt,
                  "q": qq if qq is not None else np.zeros(0),
                  "normals": nrm if nrm is not None else np.zeros(0),
                  "dipoles": dip if dip is not None else np.zeros(0), "pot": pot}
        if grad:
            arrays["grad"] = R.direct(problem, xs, qq, xt, k=k, normals=nrm, dipoles=dip,
                                      grad=True)
        for a, v in arrays.items():
            out[f"{name}_{a}"] = v
    path = os.path.join(HERE, "direct_sums.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
