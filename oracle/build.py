"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/fsl_oracle.cpp`` into ``oracle/liboracle_fsl.so`` with g++,
OpenMP, and ``-ffp-contract=off`` (the cell-index formulas of the reference
must not be fused into multiply-adds).  Also exposes ``build_ref()``, which
builds the reference's own Stokes-limit sources for the host into
``oracle/_ref/`` when the reference tree is present (see ``ref_cpu/``).

Two more builds of the same source serve the CPU baseline timings:
``real="f32"`` replaces the arithmetic type ``double`` by ``float`` throughout
(the reference's own single-precision route is the same textual substitution
of its sources, tools/scriptFloat), and ``native=True`` compiles for the host
it runs on (``-march=native``; built where it is used, since the library
travels between machines).  Portable builds use ``-march=x86-64-v3``.
"""
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_fsl.so")
SRC = os.path.join(HERE, "fsl_oracle.cpp")
HDR = os.path.join(HERE, "fsl_oracle.h")

CXXFLAGS = ["-O3", "-fopenmp", "-ffp-contract=off", "-fPIC",
            "-shared", "-std=c++17", "-Wall", "-Wno-unused-function"]


def lib_path(real="f64", native=False):
    return os.path.join(HERE, "liboracle_fsl" + ("_f32" if real == "f32" else "")
                        + ("_native" if native else "") + ".so")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force=False, real="f64", native=False):
    lib = lib_path(real, native)
    if not (force or _stale(lib, [SRC, HDR])):
        return lib
    arch = ["-march=native"] if native else ["-march=x86-64-v3"]
    with tempfile.TemporaryDirectory() as tmpdir:
        src = SRC
        if real == "f32":
            for f in (SRC, HDR):
                with open(f) as fh:
                    text = re.sub(r"\bdouble\b", "float", fh.read())
                with open(os.path.join(tmpdir, os.path.basename(f)), "w") as fh:
                    fh.write(text)
            src = os.path.join(tmpdir, os.path.basename(SRC))
        tmp = lib + ".tmp"
        subprocess.run(["g++"] + CXXFLAGS + arch + [src, "-o", tmp], check=True)
        os.replace(tmp, lib)
    return lib


def build_ref(force=False):
    """Build oracle/_ref from the reference sources if they are mounted here."""
    sys.path.insert(0, os.path.join(HERE, "ref_cpu"))
    try:
        import build_ref as br  # noqa: E402
    finally:
        sys.path.pop(0)
    return br.build(force=force)


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_oracle(force="--force" in sys.argv, real="f32"))
