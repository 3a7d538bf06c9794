"""The allocation-free Morton sort (wbfmm_b200_morton_sort_noalloc).

Callers that cannot allocate device memory where they need the tree's point
ordering -- serving loops that must not take cudaMalloc's device-wide
synchronisation, processes whose GPU memory belongs to another allocator --
use this entry point with their own buffers; its scratch is a fixed device
array inside the library.  Its permutation must equal the one the allocating
path (wbfmm_b200_set_sources) computes, call after call; sizes beyond the
fixed scratch must be refused; a point on the cube's boundary must be
reported, and the next good call must not see the stale flag; and a call
must leave the device's free memory unchanged.

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


def _call(f, p, dev, xs=None):
    import torch

    xs = p.xs if xs is None else xs
    n = xs.shape[0]
    pts = torch.from_numpy(np.ascontiguousarray(xs)).to(dev)
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    ip = torch.empty(n, dtype=torch.int32, device=dev)
    x0 = np.ascontiguousarray(p.x0, dtype=np.float64)
    rc = f(n, pts.data_ptr(), 3, x0.ctypes.data, p.D, keys.data_ptr(), ip.data_ptr(),
           torch.cuda.current_stream(dev).cuda_stream)
    return rc, keys, ip


def test_noalloc_sort_matches_allocating_path_twice(gpu_lib):
    import torch

    f = _noalloc(gpu_lib)
    dev = torch.device("cuda", 0)
    for seed, n in ((71, 200_000), (72, 33_333)):   # two calls in a row
        p = W.laplace_cube(n, 10, depth=3, order=3, seed=seed)
        expect = _reference_order(p)
        rc, keys, ip = _call(f, p, dev)
        assert rc == 0, gpu_lib.wbfmm_b200_last_error()
        got = ip.cpu().numpy().astype(np.uint32)
        assert np.array_equal(got, expect)
        k = keys.cpu().numpy().view(np.uint64)
        assert np.all(k[1:] >= k[:-1])


def test_noalloc_sort_reports_domain_then_recovers(gpu_lib):
    """A point on a face of the cube is refused (strict interior, as the
    tree build); the next call with valid points succeeds, so the shared
    flag was cleared in between."""
    import torch

    f = _noalloc(gpu_lib)
    dev = torch.device("cuda", 0)
    p = W.laplace_cube(5_000, 10, depth=3, order=3, seed=73)
    bad = p.xs.copy()
    bad[17, 1] = p.x0[1]
    rc, _, _ = _call(f, p, dev, bad)
    assert rc == -2, gpu_lib.wbfmm_b200_last_error()
    rc, _, ip = _call(f, p, dev)
    assert rc == 0, gpu_lib.wbfmm_b200_last_error()
    assert np.array_equal(ip.cpu().numpy().astype(np.uint32), _reference_order(p))


def test_noalloc_sort_leaves_device_memory_unchanged(gpu_lib):
    """After a first call (module loading and the scratch lookup happen
    there), further calls change neither torch's allocations nor the
    device's free memory."""
    import torch

    f = _noalloc(gpu_lib)
    dev = torch.device("cuda", 0)
    p = W.laplace_cube(100_000, 10, depth=3, order=3, seed=74)
    pts = torch.from_numpy(np.ascontiguousarray(p.xs)).to(dev)
    keys = torch.empty(p.ns, dtype=torch.int64, device=dev)
    ip = torch.empty(p.ns, dtype=torch.int32, device=dev)
    x0 = np.ascontiguousarray(p.x0, dtype=np.float64)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def once():
        return f(p.ns, pts.data_ptr(), 3, x0.ctypes.data, p.D, keys.data_ptr(),
                 ip.data_ptr(), stream)

    assert once() == 0
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    alloc0 = torch.cuda.memory_allocated(dev)
    for _ in range(3):
        assert once() == 0
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert torch.cuda.memory_allocated(dev) == alloc0


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
