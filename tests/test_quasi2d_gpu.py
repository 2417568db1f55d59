"""The quasi-2D family (keywords quasi2D and stokesLimit2D) on the GPU
against the reference's own outputs (tests/golden/q2d_*, s2d_*) and the FP64
oracle.  The family is FP64 throughout on both sides; stated tolerance:
1e-9 of the displacement (max |gpu - ref| / max |ref displacement|)."""
import numpy as np
import pytest

import golden_cases as G
from helpers import rel_inf

pytestmark = pytest.mark.gpu

TOL = 1e-9
CASES = [n for n in G.cases() if n.startswith(("q2d_", "s2d_"))]


def _gpu_for(fsl, c):
    g = fsl.StokesLimit(c["cfg"], c["q0"])
    if c["bonds"] is not None:
        b = c["bonds"]
        g.load_bonds(b["bi"], b["bj"], b["k"], b["r0"], b["fi"], b["fk"], b["fr0"], b["fxyz"])
    return g


@pytest.mark.parametrize("name", CASES)
def test_gpu_reproduces_reference(fsl, name):
    c = G.load(name)
    g = _gpu_for(fsl, c)
    done = 0
    for step, taken in G.sample_steps(c["run"], c["cfg"].scheme):
        g.step(taken - done)
        done = taken
        g.sync()
        t = step * c["cfg"].dt
        key = min(c["pos"], key=lambda x: abs(x - t))
        ref = c["pos"][key] - c["q0"]
        got = g.positions() - c["q0"]
        # the text files hold 15 significant digits of |q| ~ L/2
        floor = 1e-13 * np.abs(c["pos"][key]).max() * 10
        assert np.abs(got - ref).max() <= max(floor, TOL * np.abs(ref).max()), (name, step)
    g.close()


@pytest.mark.parametrize("name", CASES)
def test_gpu_tracks_oracle_velocity(fsl, oracle, name):
    """Field and positions after two steps against the oracle."""
    c = G.load(name)
    cfg = c["cfg"]
    g = _gpu_for(fsl, c)
    o = oracle.Oracle(cfg.mx, cfg.my, cfg.mz, cfg.lx, cfg.ly, cfg.lz, c["q0"], eta=cfg.shearviscosity,
                      kT=cfg.temperature, dt=cfg.dt, cutoff=cfg.cutoff, pair=cfg.pair,
                      nonbonded=cfg.nonbonded, seed=c["seed"], scheme=cfg.scheme, radius=cfg.radius,
                      ndrift=cfg.ndrift, use_rfd=cfg.use_rfd, predictor_corrector=cfg.predictor_corrector,
                      saffman_kc=cfg.saffman_kc, saffman_width=cfg.saffman_width, shear_amp=cfg.shear_amp)
    if c["bonds"] is not None:
        b = c["bonds"]
        o.set_bonds(b["bi"], b["bj"], b["k"], b["r0"], b["fi"], b["fk"], b["fr0"], b["fxyz"])
    g.step(2)
    o.step(2)
    g.sync()
    assert rel_inf(g.velocity64(), o.velocity()) < TOL
    assert rel_inf(g.positions() - c["q0"], o.positions() - c["q0"]) < TOL
    g.close()


def test_batch_of_2d_variants_equals_alone(fsl):
    """Two variants of the family and a 3-D instance in one batch agree with
    their lone runs (FP64 atomics: within the stated tolerance)."""
    cs = [G.load(n) for n in ("q2d_rpy_lattice", "s2d_saffman_shear")]
    alone = []
    for c in cs:
        g = _gpu_for(fsl, c)
        g.step(3)
        g.sync()
        alone.append(g.positions())
        g.close()
    b = fsl.Batch([c["cfg"] for c in cs], [c["q0"] for c in cs])
    b.step(3)
    b.sync()
    for i, c in enumerate(cs):
        assert rel_inf(b.positions(i) - c["q0"], alone[i] - c["q0"]) < TOL
    b.close()
