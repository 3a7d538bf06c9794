"""Build libwbfmm_b200.so in-tree for sm_100a.

CUDA sources in wbfmm_b200/csrc/*.cu are compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the drop-in
wbfmm.h layer (wbfmm_b200/csrc/wbfmm_api.c) is plain C compiled with gcc; all
objects link into one shared library next to this file.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwbfmm_b200.so")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-Xcompiler", "-O3", "-I", CSRC, "-I", INCLUDE]
CFLAGS = ["-O2", "-fPIC", "-std=c11", "-Wall", "-I", INCLUDE, "-I", CSRC]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    c = sorted(f for f in os.listdir(CSRC) if f.endswith(".c"))
    return cu, c


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
          if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    cu, c = _sources()
    hdrs = _headers()
    jobs = []
    objs = []
    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, __file__] + hdrs):
            jobs.append([NVCC, *NVFLAGS, "-c", src, "-o", obj])
    for f in c:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f[:-2] + ".c.o")
        objs.append(obj)
        if force or _stale(obj, [src, __file__] + hdrs):
            jobs.append(["gcc", *CFLAGS, "-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for out in ex.map(_run, jobs):
                if verbose and out.strip():
                    print(out)
    if force or jobs or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
