"""Build recipe of libfluamsl.so and the `fluam` executable (sm_100a).

All CUDA sources are compiled with nvcc for ``-gencode arch=compute_100a,
code=sm_100a`` and linked in-tree into ``fluam_b200/libfluamsl.so``; the
drop-in executable ``fluam_b200/fluam`` links against it with an $ORIGIN
rpath.  Nothing is installed outside the repository.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfluamsl.so")
EXE = os.path.join(HERE, "fluam")

CU_SOURCES = ["fsl_particles.cu", "fsl_fft.cu", "fsl_group.cu", "fsl_api.cu", "fsl_batch.cu", "fsl_server.cu", "fsl_noalloc.cu",
              "fsl_fp64.cu", "fsl_q2d.cu", "fsl_inc.cu"]
CPP_SOURCES = ["fsl_datamain.cpp"]
HEADERS = ["fsl_internal.cuh", "fsl_group.cuh", "fsl_fft_reg.cuh", "fsl_fft_lines.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-Wall", "--expt-relaxed-constexpr"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "fluamsl.h")]
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs):
            flags = list(NVCC_FLAGS)
            if ptxas_info and src.endswith(".cu"):
                flags += ["-Xptxas", "-v"]
            if src.endswith(".cpp"):
                flags += ["-x", "cu"]
            cmd = [nvcc()] + flags + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        subprocess.run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"], check=True)
        os.replace(tmp, LIB)
    main_src = os.path.join(CSRC, "fluam_main.cpp")
    if force or _stale(EXE, [LIB, main_src]):
        tmp = EXE + ".tmp"
        subprocess.run(["g++", "-O2", "-o", tmp, main_src, "-L" + HERE, "-lfluamsl",
                        "-Wl,-rpath,$ORIGIN"], check=True)
        os.replace(tmp, EXE)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
