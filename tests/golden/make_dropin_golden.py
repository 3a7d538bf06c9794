"""Generate tests/golden/dropin_cases.npz: what a wbfmm.h client program
(tests/dropin/driver.c) sees when it runs against the unmodified reference.

Run here (where the reference sources exist):
    python tests/golden/make_dropin_golden.py

For every case of tests/dropin/harness.py:cases() the fixture keeps the field
array, t->ip, every box's {i, n}, and for each level's coefficient array its
2-norm and 16 seeded random projections (the full arrays are megabytes).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "dropin"))

import harness as H  # noqa: E402
from oracle.build_oracle import build_reference  # noqa: E402

OUT = os.path.join(HERE, "dropin_cases.npz")


def projections(a: np.ndarray) -> np.ndarray:
    r = np.random.default_rng(7).standard_normal((16, a.size))
    return r @ a


def summarise(name: str, c: H.Case, out: dict) -> dict:
    d = {f"{name}/f": out["f"], f"{name}/ip": out["ip"]}
    d[f"{name}/boxes"] = np.concatenate([out[f"boxes{l}"] for l in range(c.depth + 1)])
    for l in range(1, c.depth + 1):
        for kind in ("mps", "mpr"):
            a = out[f"{kind}{l}"]
            d[f"{name}/{kind}{l}_norm"] = np.array(np.linalg.norm(a))
            d[f"{name}/{kind}{l}_proj"] = projections(a)
    return d


def main():
    if build_reference() is None or H.build_driver("reference") is None:
        raise SystemExit("reference sources not found; cannot generate fixtures")
    fixture = {}
    for name, c in H.cases().items():
        fixture.update(summarise(name, c, H.run("reference", c)))
        print(name, "done")
    np.savez_compressed(OUT, **fixture)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
