"""The incompressible fluctuating fluid (keyword incompressible) on the GPU
against the reference's own outputs (tests/golden/inc_*) and the FP64
oracle.  FP64 on both sides; stated tolerance 1e-11 of the field."""
import os
import subprocess

import numpy as np
import pytest

import golden_cases as G
from helpers import rel_inf

pytestmark = pytest.mark.gpu

TOL = 1e-11
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FLUAM = os.path.join(ROOT, "fluam_b200", "fluam")


def _gpu(fsl, c):
    g = fsl.StokesLimit(c["cfg"], np.zeros((3, 0)))
    g.set_velocity64(np.repeat(np.asarray(c["v0"])[:, None], c["nc"], axis=1))
    return g


@pytest.mark.parametrize("name", G.fluid_cases())
def test_gpu_reproduces_reference_field(fsl, name):
    c = G.load_fluid(name)
    g = _gpu(fsl, c)
    g.step(c["run"]["numsteps"] + c["run"]["numstepsRelaxation"])
    g.sync()
    v = g.velocity64().reshape(3, -1)
    assert rel_inf(v, c["v"]) < TOL
    g.close()


@pytest.mark.parametrize("name", G.fluid_cases())
def test_dropin_writes_reference_files(tmp_path, name):
    c = G.load_fluid(name)
    (tmp_path / "data.main").write_text(open(os.path.join(c["dir"], "data.main")).read())
    r = subprocess.run([FLUAM, "data.main"], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 1, r.stdout + r.stderr
    assert "INCOMPRESSIBLE" in r.stdout
    v = G.read_fluid_final(str(tmp_path / "out.fluidFinalConfiguration"), c["nc"])
    assert rel_inf(v, c["v"]) < TOL
    head = (tmp_path / "out.fluidFinalConfiguration").read_text().split("\n")[:13]
    assert head == open(os.path.join(c["dir"], "out.fluidFinalConfiguration")).read().split("\n")[:13]
    # the temperature diagnostic: same words, numbers within the tolerance
    got = (tmp_path / "out.temperature").read_text().split()
    ref = c["temperature"].split()
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        try:
            fa, fb = float(a), float(b)
        except ValueError:
            assert a == b
            continue
        assert abs(fa - fb) <= 1e-9 * max(abs(fb), 1e-6), (a, b)


def test_random_start_tracks_oracle(fsl, oracle):
    """A non-uniform start: the projection and three steps against the oracle."""
    cfg = fsl.make_config((12, 10, 8), (12.0, 10.0, 8.0), eta=0.9, kT=0.2, dt=0.05, seed=21,
                          scheme=fsl.SCHEME_INCOMPRESSIBLE, density=1.1)
    nc = 12 * 10 * 8
    v0 = np.random.default_rng(4).standard_normal((3, nc)) * 0.3
    g = fsl.StokesLimit(cfg, np.zeros((3, 0)))
    g.set_velocity64(v0)
    o = oracle.Oracle(12, 10, 8, 12.0, 10.0, 8.0, np.zeros((3, 0)), eta=0.9, kT=0.2, dt=0.05, seed=21,
                      scheme=oracle.SCHEME_INCOMPRESSIBLE, density=1.1)
    o.set_velocity(v0)
    assert rel_inf(g.velocity64().reshape(3, -1), o.velocity().reshape(3, -1)) < TOL
    g.step(3)
    o.step(3)
    g.sync()
    assert rel_inf(g.velocity64().reshape(3, -1), o.velocity().reshape(3, -1)) < TOL
    g.close()
