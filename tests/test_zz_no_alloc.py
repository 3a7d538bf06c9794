"""The allocation-free Morton sort (wbfmm_b200_morton_sort_noalloc).

Callers that cannot allocate device memory where they need the tree's point
ordering -- work recorded in a CUDA stream capture, serving loops that must
not take cudaMalloc's device-wide synchronisation, processes whose GPU memory
belongs to another allocator -- use this entry point with their own buffers;
its scratch is a fixed device array inside the library.  Its permutation must
equal the one the allocating path (wbfmm_b200_set_sources) computes, call
after call, and sizes beyond the fixed scratch must be refused.

This file is collected last so that a failure here comes after every other
test has run.
"""
import ctypes as C

import numpy as np
import pytest

from wbfmm_b200 import engine, workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.wbfmm_b200_morton_sort_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_void_p,
                  C.c_void_p, C.c_void_p]
    return f


def _reference_order(p):
    cfg = engine.SolverConfig.from_problem(p)
    with engine.Solver(cfg) as s:
        s.set_sources(p.xs)
        ip, _, _ = s.tree(0)
    return ip


def test_noalloc_sort_matches_allocating_path_twice(gpu_lib):
    import torch

    f = _noalloc(gpu_lib)
    dev = torch.device("cuda", 0)
    for seed, n in ((71, 200_000), (72, 33_333)):   # two calls in a row
        p = W.laplace_cube(n, 10, depth=3, order=3, seed=seed)
        expect = _reference_order(p)
        pts = torch.from_numpy(np.ascontiguousarray(p.xs)).to(dev)
        keys = torch.empty(n, dtype=torch.int64, device=dev)
        ip = torch.empty(n, dtype=torch.int32, device=dev)
        x0 = np.ascontiguousarray(p.x0, dtype=np.float64)
        rc = f(n, pts.data_ptr(), 3, x0.ctypes.data, p.D, keys.data_ptr(), ip.data_ptr(),
               torch.cuda.current_stream(dev).cuda_stream)
        assert rc == 0, gpu_lib.wbfmm_b200_last_error()
        got = ip.cpu().numpy().astype(np.uint32)
        assert np.array_equal(got, expect)
        k = keys.cpu().numpy().view(np.uint64)
        assert np.all(k[1:] >= k[:-1])


def test_noalloc_sort_rejects_oversize(gpu_lib):
    import torch

    f = _noalloc(gpu_lib)
    n = (1 << 20) + 1
    dev = torch.device("cuda", 0)
    pts = torch.zeros((1, 3), dtype=torch.float64, device=dev)
    x0 = np.zeros(3)
    rc = f(n, pts.data_ptr(), 3, x0.ctypes.data, 1.0, pts.data_ptr(), pts.data_ptr(), None)
    assert rc == -1
    assert b"scratch" in gpu_lib.wbfmm_b200_last_error()
