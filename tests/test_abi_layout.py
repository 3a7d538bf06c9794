"""The ctypes mirrors of the engine ABI's structs (wbfmm_b200/engine.py)
have the C layout of include/wbfmm_b200.h: every member at the offset the C
compiler gives it, and the same total size (CPU only: gcc on the header)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from wbfmm_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def c_layout(tmp_path, struct, members):
    src = tmp_path / "layout.c"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "wbfmm_b200.h"',
             "int main(void) {",
             f'  printf("size %zu\\n", sizeof({struct}));']
    for m in members:
        lines.append(f'  printf("{m} %zu\\n", offsetof({struct}, {m}));')
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
@pytest.mark.parametrize("py, cname", [(engine.Config, "wbfmm_b200_config_t"),
                                       (engine.Request, "wbfmm_b200_request_t")])
def test_struct_layout_matches_header(tmp_path, py, cname):
    names = [f[0] for f in py._fields_]
    got = c_layout(tmp_path, cname, names)
    assert got["size"] == C.sizeof(py)
    for n in names:
        assert got[n] == getattr(py, n).offset, n
