"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/fsl_oracle.cpp`` into ``oracle/liboracle_fsl.so`` with g++,
OpenMP, and ``-ffp-contract=off`` (the cell-index formulas of the reference
must not be fused into multiply-adds).  Also exposes ``build_ref()``, which
builds the reference's own Stokes-limit sources for the host into
``oracle/_ref/`` when the reference tree is present (see ``ref_cpu/``).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_fsl.so")
SRC = os.path.join(HERE, "fsl_oracle.cpp")
HDR = os.path.join(HERE, "fsl_oracle.h")

CXXFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-ffp-contract=off", "-fPIC",
            "-shared", "-std=c++17", "-Wall", "-Wno-unused-function"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force=False):
    if force or _stale(LIB, [SRC, HDR]):
        tmp = LIB + ".tmp"
        cmd = ["g++"] + CXXFLAGS + [SRC, "-o", tmp]
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


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
