"""The reference-side binding of INTEGRATION.md section 2 compiles against the
reference's own headers (where its sources are present; skipped elsewhere),
and the directed bond entries it hands over are the ones the library's
reader of the old bond-file format produces.

No GPU: the snippet is compiled with -fsyntax-only, and the bond check runs
the expansion of the reference's per-particle lists in Python against the
entries of a golden bond file.
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_sources():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_build_ref", os.path.join(ROOT, "oracle", "ref_cpu", "build_ref.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REF_SRC


def _binding_snippet():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    sec = text[text.index("## 2."):text.index("## 3.")]
    m = re.search(r"```cpp\n(.*?)```", sec, re.S)
    assert m, "no C++ block in section 2"
    return m.group(1)


def test_binding_compiles_against_reference_headers(tmp_path):
    ref_src = _reference_sources()
    if not os.path.isdir(ref_src):
        pytest.skip("reference sources not present here")
    src = tmp_path / "schemeStokesLimit_b200.cpp"
    src.write_text(_binding_snippet())
    shim = os.path.join(ROOT, "oracle", "ref_cpu", "cuda_host_shim.h")
    cmd = ["g++", "-std=gnu++14", "-fpermissive", "-w", "-fsyntax-only", "-x", "c++",
           "-include", shim, "-I", ref_src, "-I", os.path.join(ROOT, "include"), str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_binding_hands_over_the_old_format_entries():
    """The reference's per-particle lists of the old-format golden file
    (src/initializeBondedForcesOldVersion.cpp: offset of a particle = position
    of its first line, count = its lines), expanded as the binding does,
    give back the file's lines in order: what fsl_load_bonds_directed gets
    from the drop-in's reader of the same file."""
    path = os.path.join(ROOT, "tests", "golden", "bonds_old_format", "bonds.dat")
    with open(path) as f:
        n = int(f.readline())
        lines = [f.readline().split() for _ in range(n)]
    i1 = np.array([int(x[0]) for x in lines])
    i2 = np.array([int(x[1]) for x in lines])
    k = np.array([float(x[2]) for x in lines])
    r0 = np.array([float(x[3]) for x in lines])
    npart = int(max(i1.max(), i2.max())) + 1
    count = np.zeros(npart, int)
    offset = np.zeros(npart, int)
    prev = -1
    for e, a in enumerate(i1):
        if a != prev:
            offset[a] = e
        count[a] += 1
        prev = a
    bi, bj, kk, rr = [], [], [], []
    for i in range(npart):
        for e in range(count[i]):
            at = offset[i] + e
            bi.append(i)
            bj.append(i2[at])
            kk.append(k[at])
            rr.append(r0[at])
    np.testing.assert_array_equal(bi, i1)
    np.testing.assert_array_equal(bj, i2)
    np.testing.assert_array_equal(kk, k)
    np.testing.assert_array_equal(rr, r0)
    # a spring listed from one end only is one entry, not a bond of both
    pairs = set(zip(i1.tolist(), i2.tolist()))
    assert any((b, a) not in pairs for a, b in pairs)
