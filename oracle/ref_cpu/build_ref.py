"""Build recipe: the reference's own Stokes-limit path for the host.

TEST INFRASTRUCTURE ONLY.  Compiles fluam's sources where they lie
(/root/reference/src, read-only) with g++ against ``cuda_host_shim.h`` into
``oracle/_ref/fluam_ref``: the reference's `main()`, data.main parser, set-up,
time loop, kernels and output writers, executed serially on the CPU.  It is
the pin of the FP64 oracle (tests/test_oracle_vs_ref.py) and the generator of
the golden files under tests/golden/.

Two mechanical steps happen on copies written to ``oracle/_ref/src`` (never
committed): kernel launches ``k<<<g, b>>>(args)`` become
``SHIM_LAUNCH(g, b, k(args))``, because g++ cannot parse the launch syntax;
nothing else in the sources is changed.  Schemes of fluam other than
stokesLimit are not compiled; `main()`'s calls to them resolve to stubs that
report "not built" and fail.
"""
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")
SRC_OUT = os.path.join(OUT, "src")
REF = os.environ.get("FLUAM_REFERENCE", "/root/reference")
REF_SRC = os.path.join(REF, "src")
EXE = os.path.join(OUT, "fluam_ref")

# The GPU translation unit of the reference (src/GPU.cu) includes ~200 files;
# these are the ones the stokesLimit scheme uses, in GPU.cu's order.
GPU_FILES = [
    "gpuVariables.cu", "moduGPU.cu", "texturesCells.cu", "initializeVecinosGPU.cu",
    "randomNumbers.cu", "allocateErrorArray.cu", "deltaGPU.cu", "initParticlesInCell.cu",
    "initializeNeighborsGPU.cu", "texturesBoundaries.cu", "forceBoundaryGPU.cu",
    "initForcesNonBonded.cu", "createBondedForcesGPU.cu", "freeBondedForcesGPU.cu",
    "forceBondedGPU.cu", "initializePrefactorFourierSpace.cu",
    "initializeFluidIncompressibleGPU.cu", "realToComplex.cu", "createBoundariesRK2GPU.cu",
    "freeBoundariesRK2GPU.cu", "createCellsStokesLimitGPU.cu", "freeCellsStokesLimitGPU.cu",
    "stokesLimitFunctions.cu", "boundaryParticlesFunctionStokesLimit.cu",
    "saveFunctionsSchemeStokesLimit.cu", "gpuToHostStokesLimit.cu", "runSchemeStokesLimit.cu",
    "boundaryParticlesFunctionStokesLimitFirstOrder.cu", "runSchemeStokesLimitFirstOrder.cu",
    # the quasi-2D / stokesLimit2D family (src/GPU.cu:197, 279-287)
    "quasiNeutrallyBuoyantFunctions2D.cu", "createCellsQuasi2DGPU.cu", "freeCellsQuasi2DGPU.cu",
    "createBoundariesQuasi2DGPU.cu", "freeBoundariesQuasi2DGPU.cu", "quasi2DFunctions.cu",
    "texturesCellsQuasi2D.cu", "runSchemeQuasi2D.cu",
    # the incompressible scheme (src/GPU.cu:158-171)
    "projectionDivergenceFree.cu", "saveFunctionsSchemeIncompressible.cu",
    "createCellsIncompressibleGPU.cu", "freeCellsIncompressibleGPU.cu", "gpuToHostIncompressible.cu",
    "kernelConstructW.cu", "kernelUpdateVIncompressible.cu", "runSchemeIncompressible.cu",
]
GPU_HEADERS = ["header.h", "cells.h", "fluid.h", "boundary.h", "headerOtherFluidVariables.h",
               "particles.h", "hydroAnalysis.h"]
# Host translation units of the path (each compiled on its own, as the
# reference's Makefile does).
HOST_FILES = [
    "main.cpp", "loadDataMain.cu", "cudaDevice.cu", "initializeRandomNumber.cpp", "rantest.cu",
    "gauss.cu", "schemeStokesLimit.cu", "schemeStokesLimitFirstOrder.cu", "schemeQuasi2D.cu",
    "schemeIncompressible.cu", "temperature.cu", "saveFluidFinalConfiguration.cu",
    "createCells.cpp", "createParticles.cpp",
    "simpleCubic.cpp", "initializeBondedForces.cpp", "initializeBondedForcesOldVersion.cpp",
    "initializeFluid.cpp", "modu.cu",
    "saveSeed.cpp", "saveTime.cpp", "saveParticles.cu", "freeParticles.cu", "random_frenk.cu",
]

CXX = ["g++", "-O2", "-std=gnu++14", "-fpermissive", "-w", "-ffp-contract=off", "-fPIC"]

_LAUNCH = re.compile(r"([A-Za-z_]\w*)\s*<<<")


def _split_top(s):
    depth, out, cur = 0, [], ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    out.append(cur)
    return out


def rewrite_launches(text):
    """k<<<g, b>>>(args) -> SHIM_LAUNCH((g), (b), k(args))"""
    out, pos = [], 0
    while True:
        m = _LAUNCH.search(text, pos)
        if not m:
            out.append(text[pos:])
            break
        out.append(text[pos:m.start()])
        end_cfg = text.index(">>>", m.end())
        cfg = _split_top(text[m.end():end_cfg])
        j = text.index("(", end_cfg)
        depth, k = 0, j
        while True:
            if text[k] == "(":
                depth += 1
            elif text[k] == ")":
                depth -= 1
                if depth == 0:
                    break
            k += 1
        args = text[j + 1:k]
        out.append(f"SHIM_LAUNCH(({cfg[0].strip()}), ({cfg[1].strip()}), {m.group(1)}({args}))")
        pos = k + 1
    return "".join(out)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not os.path.isdir(REF_SRC):
        raise RuntimeError(f"reference sources not found at {REF_SRC}")
    os.makedirs(SRC_OUT, exist_ok=True)
    for f in GPU_FILES + HOST_FILES:
        src = os.path.join(REF_SRC, f)
        dst = os.path.join(SRC_OUT, f)
        if force or _stale(dst, [src, __file__]):
            with open(src, errors="replace") as fh:
                text = fh.read()
            with open(dst, "w") as fh:
                fh.write(rewrite_launches(text))
    # the oracle library provides the Philox noise that replaces cuRAND
    sys.path.insert(0, ORACLE)
    try:
        import build as ob  # oracle/build.py
        orc = ob.build_oracle()
    finally:
        sys.path.pop(0)
    shim = os.path.join(HERE, "cuda_host_shim.h")
    inc = ["-include", shim, "-I", SRC_OUT, "-I", REF_SRC, "-I", ORACLE]
    objs = []
    units = [(os.path.join(HERE, "ref_gpu_tu.cpp"), "gpu_tu.o"),
             (os.path.join(HERE, "shim_impl.cpp"), "shim_impl.o"),
             (os.path.join(HERE, "ref_stubs.cpp"), "ref_stubs.o")]
    units += [(os.path.join(SRC_OUT, f), f + ".o") for f in HOST_FILES]
    deps_common = [shim, __file__] + [os.path.join(SRC_OUT, f) for f in GPU_FILES]
    for src, obj in units:
        o = os.path.join(OUT, obj)
        objs.append(o)
        if force or _stale(o, [src] + deps_common):
            cmd = CXX + ["-x", "c++"] + inc + ["-c", src, "-o", o]
            if os.path.basename(src) in HOST_FILES:
                # host set-up and I/O code, not on the timed path; at -O0 the
                # value-returning functions without a return statement
                # (freeBondedForces, src/initializeBondedForces.cpp:186-207)
                # return garbage instead of being compiled as unreachable
                cmd.insert(-4, "-O0")  # after -O2: the last -O flag wins
            if os.path.basename(src) == "initializeBondedForces.cpp":
                # freeBondedForces has no return statement (undefined
                # behaviour; g++ 13 traps there at the end of every bonded
                # run); its definition is renamed and ref_stubs.cpp links one
                # that returns 1
                cmd.insert(-4, "-DfreeBondedForces=fluam_ref_freeBondedForces_no_return")
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(EXE, objs + [orc]):
        subprocess.run(["g++", "-o", EXE] + objs + [orc, "-Wl,-rpath," + ORACLE], check=True)
    return EXE


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
