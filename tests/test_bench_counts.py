"""The benchmark's algorithmic M2L pair counts (the roofline's numerator)
against a direct enumeration of list 4 on small trees: every pair of a
dense level, the pairs of the boxes that hold targets, and of those only the
pairs whose source box holds sources (the work of a skip_empty solve, whose
kernels skip empty source boxes).  List 4 of a box: the children of its
parent's neighbours that are not its own neighbours (src/indexing.c)."""
import itertools
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _boxes(pts, level):
    n = 1 << level
    return {tuple(b) for b in np.clip(np.floor(np.asarray(pts) * n).astype(int), 0, n - 1)}


def _list4(b, level):
    n = 1 << level
    out = []
    for c in itertools.product(range(n), repeat=3):
        parent_near = all(abs(c[d] // 2 - b[d] // 2) <= 1 for d in range(3))
        near = all(abs(c[d] - b[d]) <= 1 for d in range(3))
        if parent_near and not near:
            out.append(c)
    return out


@pytest.mark.parametrize("level", [2, 3, 4])
def test_list4_pair_counts(level):
    rng = np.random.default_rng(level)
    xs = rng.random((250, 3)) ** 2          # uneven: many empty boxes
    xt = rng.random((150, 3))
    tb, sb = _boxes(xt, level), _boxes(xs, level)
    all_pairs = sum(len(_list4(b, level)) for b in tb)
    src_pairs = sum(sum(c in sb for c in _list4(b, level)) for b in tb)
    assert bench.list4_pairs_at(xt, [0, 0, 0], 1.0, level) == all_pairs
    assert bench.list4_pairs_at(xt, [0, 0, 0], 1.0, level, xs) == src_pairs
    if level <= 3:
        dense = sum(len(_list4(b, level)) for b in itertools.product(range(1 << level), repeat=3))
        assert bench.list4_pairs(level)[level] == dense
