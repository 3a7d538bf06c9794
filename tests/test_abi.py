"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "wbfmm_b200", "libwbfmm_b200.so")


def declared_functions():
    names = set()
    for f in os.listdir(INCLUDE):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = text.replace("\\\n", " ")
        text = re.sub(r"#define[^\n]*", "", text)
        for m in re.finditer(r"\b(wbfmm_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        pytest.fail(f"{LIB} not built (run python -m wbfmm_b200.build)")
    return ctypes.CDLL(LIB)


def test_library_exports_all_declared_symbols(lib):
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_build_targets_sm100a():
    from wbfmm_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVFLAGS)


def test_error_reporting_without_gpu(lib):
    lib.wbfmm_b200_last_error.restype = ctypes.c_char_p
    lib.wbfmm_b200_device_count.restype = ctypes.c_int
    n = lib.wbfmm_b200_device_count()
    assert n >= 0
    if n == 0:
        lib.wbfmm_b200_solver_create.restype = ctypes.c_int
        from wbfmm_b200 import engine
        cfg = engine.SolverConfig(engine.LAPLACE, 3, [0, 4, 4, 4], [0, 4, 4, 4]).to_c()
        h = ctypes.c_void_p()
        rc = lib.wbfmm_b200_solver_create(ctypes.byref(h), ctypes.byref(cfg), None)
        assert rc == -7
        assert b"no CUDA device" in lib.wbfmm_b200_last_error()
