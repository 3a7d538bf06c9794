"""Build recipe for the test oracle (test infrastructure only).

Two shared libraries come out of here:

* ``oracle/liboracle.so`` -- the CPU restatement in ``oracle/wbfmm_oracle.c``
  (our own code; builds anywhere gcc is present);
* ``oracle/_ref/libwbfmm_ref.so`` -- the UNMODIFIED reference sources from
  ``/root/reference/src`` plus the GLib/blaswrap shim in ``oracle/shim`` and
  the call-sequence harness ``oracle/ref_harness.c``.  Built only where the
  reference tree is present; the built ``.so`` travels with the repository
  snapshot (``oracle/_ref`` is git-ignored, not snapshot-ignored).

Flags follow the reference's own build (configure.ac, tools/Makefile.am):
``-O3 -g -mavx -mfma -fopenmp -DWBFMM_USE_AVX -DHAVE_CONFIG_H`` with its shipped
``config.h``.  The reference's logging module (src/wbfmm-logging.c) is left out:
nothing on the FMM path calls it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# where the reference tree lies in the build container: the one place this
# repository names it (WBFMM_REFERENCE_ROOT overrides)
REF_ROOT = os.environ.get("WBFMM_REFERENCE_ROOT", "/root/reference")
REF_OUT = os.path.join(HERE, "_ref")
BUILD_DIR = os.path.join(HERE, "_build")

REF_FLAGS = [
    "-O3", "-g", "-mavx", "-mfma", "-fopenmp", "-fPIC",
    "-DWBFMM_USE_AVX", "-DHAVE_CONFIG_H",
    '-DWBFMM_COMPILER_FLAGS="-O3 -g -mavx -mfma -fopenmp -DWBFMM_USE_AVX"',
]


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed: " + " ".join(cmd[:4]) + " ...")


def build_restatement(force: bool = False) -> str:
    """Compile the CPU restatement (oracle/wbfmm_oracle.c)."""
    src = os.path.join(HERE, "wbfmm_oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if force or _newer(out, [src, __file__]):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-pthread", "-ffp-contract=off",
              src, "-o", out, "-lm"])
    return out


# the sources the reference compiles a second time in single precision
# (libsub, -DWBFMM_SINGLE_PRECISION: src/Makefile.am), giving its *_f API
SINGLE_PRECISION = (
    "expansions.c", "translations.c", "rotations.c", "rotations-laplace.c", "util.c",
    "boxes.c", "shift.c", "shift-laplace.c", "shiftbw.c", "shiftbw-laplace.c", "pass.c",
    "pass-laplace.c", "laplace.c", "targets.c", "gradient.c", "gradient-laplace.c",
    "local.c", "local-laplace.c", "direct.c", "direct-laplace.c")


def build_reference(force: bool = False) -> str | None:
    """Compile the reference sources + shim + harness; None if absent.  The
    library holds both precisions, as the reference's own build does."""
    src_dir = os.path.join(REF_ROOT, "src")
    out = os.path.join(REF_OUT, "libwbfmm_ref.so")
    if not os.path.isdir(src_dir):
        return out if os.path.exists(out) else None
    srcs = sorted(
        os.path.join(src_dir, f)
        for f in os.listdir(src_dir)
        if f.endswith(".c") and f != "wbfmm-logging.c"
    )
    extra = [os.path.join(HERE, "shim", "glib_shim.c"),
             os.path.join(HERE, "ref_harness.c")]
    deps = srcs + extra + [os.path.join(HERE, "shim", "glib.h"), __file__]
    if not (force or _newer(out, deps)):
        return out
    os.makedirs(REF_OUT, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    incs = ["-I", os.path.join(HERE, "shim"), "-I", REF_ROOT, "-I", src_dir]
    for s in srcs + extra:
        o = os.path.join(BUILD_DIR, os.path.basename(s)[:-2] + ".o")
        if force or _newer(o, [s]):
            _run(["gcc", "-c", *REF_FLAGS, *incs, s, "-o", o])
        objs.append(o)
    for s in srcs:
        if os.path.basename(s) not in SINGLE_PRECISION:
            continue
        o = os.path.join(BUILD_DIR, os.path.basename(s)[:-2] + "-float.o")
        if force or _newer(o, [s]):
            _run(["gcc", "-c", *REF_FLAGS, "-DWBFMM_SINGLE_PRECISION", *incs, s, "-o", o])
        objs.append(o)
    _run(["gcc", "-shared", "-fopenmp", "-o", out, *objs, "-lm", "-lpthread"])
    return out


REPO = os.path.dirname(HERE)
# driver name -> (source in tools/, substitutions of the reference's own
# generation step: tools/make-source for double, tools/make-source-float for
# single precision)
_DOUBLE = (("WBFMM_REAL", "gdouble"), ("_FLOAT", ""), ("FLOATFMT", "lg"),
           ("FLOATEXP", "1.16e"))
_FLOAT = (("WBFMM_REAL", "gfloat"), ("_FLOAT", "_f"), ("FLOATFMT", "g"),
          ("FLOATEXP", "1.16e"))
DRIVER_SOURCES = {
    "wbfmm-tree-calc": ("wbfmm-tree-calc", _DOUBLE),
    "wbfmm-laplace-tree-calc": ("wbfmm-laplace-tree-calc", _DOUBLE),
    "wbfmm-tree-calc-float": ("wbfmm-tree-calc", _FLOAT),
    "wbfmm-laplace-tree-calc-float": ("wbfmm-laplace-tree-calc", _FLOAT),
}
DRIVERS = tuple(DRIVER_SOURCES)


def _generate_driver(src_in: str, out: str, subs=_DOUBLE) -> None:
    """The reference's own generation step for its drivers (tools/make-source,
    tools/make-source-float: names and formats of one precision)."""
    text = open(src_in).read()
    for a, b in subs:
        text = text.replace(a, b)
    with open(out, "w") as f:
        f.write(text)


def build_reference_drivers(force: bool = False) -> dict | None:
    """The reference's command-line drivers (tools/wbfmm-tree-calc.c.in,
    tools/wbfmm-laplace-tree-calc.c.in: text point files in, fields out),
    built twice from the same unmodified source: linked with the reference
    library (``<tool>-reference``) and with this repository's drop-in
    ``include/wbfmm.h`` + ``libwbfmm_b200.so`` (``<tool>-b200``).  Outputs in
    ``oracle/_ref``; None where neither the reference tree nor earlier builds
    are present."""
    tools_dir = os.path.join(REF_ROOT, "tools")
    outs = {t: (os.path.join(REF_OUT, t + "-reference"), os.path.join(REF_OUT, t + "-b200"))
            for t in DRIVERS}
    if not os.path.isdir(tools_dir):
        return outs if all(os.path.exists(b) for pair in outs.values() for b in pair) else None
    ref_lib = build_reference(force)
    b200_lib = os.path.join(REPO, "wbfmm_b200", "libwbfmm_b200.so")
    if ref_lib is None or not os.path.exists(b200_lib):
        return None
    os.makedirs(BUILD_DIR, exist_ok=True)
    shim = os.path.join(HERE, "shim", "glib_shim.c")
    shim_o = os.path.join(BUILD_DIR, "glib_shim_driver.o")
    if force or _newer(shim_o, [shim]):
        _run(["gcc", "-O2", "-I", os.path.join(HERE, "shim"), "-c", shim, "-o", shim_o])
    for t, (ref_bin, b200_bin) in outs.items():
        base, subs = DRIVER_SOURCES[t]
        src_in = os.path.join(tools_dir, base + ".c.in")
        gen = os.path.join(BUILD_DIR, t + ".c")
        if force or _newer(gen, [src_in, __file__]):
            _generate_driver(src_in, gen, subs)
        common = ["-O2", "-DHAVE_CONFIG_H", gen]
        if force or _newer(ref_bin, [gen, ref_lib]):
            _run(["gcc", *common, "-fopenmp", "-I", os.path.join(HERE, "shim"), "-I", REF_ROOT,
                  "-I", os.path.join(REF_ROOT, "src"), "-o", ref_bin, "-L", REF_OUT,
                  "-lwbfmm_ref", "-Wl,-rpath,$ORIGIN", "-lm"])
        if force or _newer(b200_bin, [gen, b200_lib, shim_o]):
            _run(["gcc", *common, "-I", os.path.join(REPO, "include"), "-I",
                  os.path.join(HERE, "shim"), "-I", REF_ROOT, shim_o, "-o", b200_bin,
                  "-L", os.path.dirname(b200_lib), "-lwbfmm_b200",
                  "-Wl,-rpath,$ORIGIN/../../wbfmm_b200", "-lm"])
    return outs


def main() -> None:
    print(build_restatement(force="--force" in sys.argv))
    print(build_reference(force="--force" in sys.argv))
    print(build_reference_drivers(force="--force" in sys.argv))


if __name__ == "__main__":
    main()
