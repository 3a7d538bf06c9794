"""The benchmark's algorithmic M2L pair counts (the roofline's numerator)
against a direct enumeration of list 4 on small trees: every pair of a
dense level, the pairs of the boxes that hold targets, and of those only the
pairs whose source box holds sources (the work of a skip_empty solve, whose
kernels skip empty source boxes).  List 4 of a box: the children of its
parent's neighbours that are not its own neighbours (src/indexing.c).  Also
the FLOPs per pair, and the DRAM traffic read from the committed ncu
summaries."""
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


@pytest.mark.parametrize("p", range(0, 21))
def test_flops_per_pair_closed_forms(p):
    """The roofline's FLOPs per list-4 pair: the closed forms of R(p) (the
    rotation's MACs, sum over degrees of (2n+1)^2) and X(p) (the coaxial
    translation's MACs, (p+1-|m|)^2 per order m) against the sums."""
    R = sum((2 * n + 1) ** 2 for n in range(p + 1))
    X = sum((p + 1 - abs(m)) ** 2 for m in range(-p, p + 1))
    assert bench.helm_flops_per_pair(p) == 2 * 4 * R + 8 * X
    assert bench.lap_flops_per_pair(p) == 2 * 2 * R + 2 * X


@pytest.mark.parametrize("path, total", [
    (bench.TILE_PROFILE, 71.904256e6 + 5.196288e6),
    (bench.TILE_HELM_PROFILE, 11.853056e6),
    (bench.P2P_PROFILE, 18.511872e6 + 222.72e3),
])
def test_profile_traffic_parses_committed_summaries(path, total):
    """The `traffic` of the bench line comes from the committed ncu
    summaries: read + write DRAM bytes, units scaled."""
    assert bench.tile_profile_traffic(path) == pytest.approx(total, rel=1e-12)


def test_profile_traffic_refuses_malformed_rows(tmp_path):
    """A summary without both rows, or with a row that is not `value unit`,
    gives no traffic rather than a wrong one."""
    good = ("| DRAM read (`dram__bytes_read.sum`) | 2.5 Mbyte |\n"
            "| DRAM write (`dram__bytes_write.sum`) | 10 Kbyte |\n")
    f = tmp_path / "p.md"
    f.write_text(good)
    assert bench.tile_profile_traffic(str(f)) == pytest.approx(2.51e6)
    f.write_text(good.splitlines()[0] + "\n")
    assert bench.tile_profile_traffic(str(f)) is None
    f.write_text("| read / write (`dram__bytes_read.sum`, `dram__bytes_write.sum`) | 1.9 GB / 0.9 GB |\n")
    assert bench.tile_profile_traffic(str(f)) is None
    assert bench.tile_profile_traffic(str(tmp_path / "missing.md")) is None
