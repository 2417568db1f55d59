"""Pin of the FP64 oracle against the reference itself.

tests/golden/ holds outputs of the reference's own stokesLimit sources
(src/stokesLimitFunctions.cu and the rest of its path) built for the host by
oracle/ref_cpu/build_ref.py; the oracle, fed the same inputs and the same
noise, must reproduce them to the precision of the 15-digit text files.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import golden_cases as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FLUAM_REF = os.path.join(ROOT, "oracle", "_ref", "fluam_ref")


def _reference_sources():
    """The reference's source tree as the build recipe finds it (the
    FLUAM_REFERENCE variable, else the recipe's default location)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_build_ref", os.path.join(ROOT, "oracle", "ref_cpu", "build_ref.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REF_SRC


def _oracle_for(oracle, c):
    cfg = c["cfg"]
    o = oracle.Oracle(cfg.mx, cfg.my, cfg.mz, cfg.lx, cfg.ly, cfg.lz, c["q0"],
                      eta=cfg.shearviscosity, kT=cfg.temperature, dt=cfg.dt, cutoff=cfg.cutoff,
                      kernel=cfg.kernel, pair=cfg.pair, soft_epsilon=cfg.soft_epsilon,
                      rfd=cfg.rfd, nonbonded=cfg.nonbonded, extra_mobility=cfg.extra_mobility,
                      seed=c["seed"], scheme=cfg.scheme, radius=cfg.radius, ndrift=cfg.ndrift,
                      use_rfd=cfg.use_rfd, predictor_corrector=cfg.predictor_corrector,
                      saffman_kc=cfg.saffman_kc, saffman_width=cfg.saffman_width,
                      shear_amp=cfg.shear_amp)
    if c["bonds"] is not None:
        b = c["bonds"]
        o.set_bonds(b["bi"], b["bj"], b["k"], b["r0"], b["fi"], b["fk"], b["fr0"], b["fxyz"],
                    directed=b["directed"])
    return o


@pytest.mark.parametrize("name", G.cases())
def test_oracle_reproduces_reference(oracle, name):
    c = G.load(name)
    o = _oracle_for(oracle, c)
    dt = c["cfg"].dt
    done = 0
    samples = G.sample_steps(c["run"], c["cfg"].scheme)
    assert len(samples) == len(c["pos"]) > 0
    for step, taken in samples:
        o.step(taken - done)
        done = taken
        t = step * dt
        key = min(c["pos"], key=lambda x: abs(x - t))
        assert abs(key - t) < 1e-12
        q_ref = c["pos"][key]
        dq_ref = q_ref - c["q0"]
        dq_orc = o.positions() - c["q0"]
        # 15 significant digits of |q| ~ L/2 bound the text's resolution
        tol = 1e-14 * np.abs(q_ref).max() * 10
        assert np.abs(dq_orc - dq_ref).max() <= max(tol, 1e-10 * np.abs(dq_ref).max()), name
        if c["frc"] is not None:
            f_ref = c["frc"][key]
            F = o.forces()
            assert np.abs(F - f_ref).max() <= 1e-12 + 1e-10 * np.abs(f_ref).max(), name


@pytest.mark.parametrize("name", G.cases())
def test_golden_files_regenerate_identically(tmp_path, name):
    """Where the reference sources are present, rerun the reference and get
    the committed fixture back byte for byte."""
    if not (os.path.exists(FLUAM_REF) and os.path.isdir(_reference_sources())):
        pytest.skip("reference host build not available here")
    src = os.path.join(G.GOLDEN, name)
    for f in os.listdir(src):
        if not f.startswith("out."):
            shutil.copy(os.path.join(src, f), tmp_path / f)
    r = subprocess.run([FLUAM_REF, "data.main"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert "END" in r.stdout, r.stdout[-1000:]
    for ext in (".particles", ".velocityParticles", ".seed"):
        mine, ref = tmp_path / ("out" + ext), os.path.join(src, "out" + ext)
        assert os.path.exists(mine) == os.path.exists(ref), ext
        if os.path.exists(ref):
            assert open(mine).read() == open(ref).read()


@pytest.mark.parametrize("name", G.fluid_cases())
def test_oracle_reproduces_reference_fluid(oracle, name):
    """The incompressible scheme: the final field of the reference (the last
    sample, here the last step) from the same uniform start and noise."""
    c = G.load_fluid(name)
    cfg = c["cfg"]
    o = oracle.Oracle(cfg.mx, cfg.my, cfg.mz, cfg.lx, cfg.ly, cfg.lz, np.zeros((3, 0)),
                      eta=cfg.shearviscosity, kT=cfg.temperature, dt=cfg.dt, seed=c["seed"],
                      scheme=oracle.SCHEME_INCOMPRESSIBLE, density=cfg.density)
    v0 = np.repeat(np.asarray(c["v0"])[:, None], c["nc"], axis=1)
    o.set_velocity(v0)
    o.step(c["run"]["numsteps"] + c["run"]["numstepsRelaxation"])
    v = o.velocity().reshape(3, -1)
    assert np.abs(v - c["v"]).max() <= 1e-12 * np.abs(c["v"]).max() * 10


@pytest.mark.parametrize("name", G.fluid_cases())
def test_fluid_golden_files_regenerate_identically(tmp_path, name):
    if not (os.path.exists(FLUAM_REF) and os.path.isdir(_reference_sources())):
        pytest.skip("reference host build not available here")
    src = os.path.join(G.GOLDEN, name)
    shutil.copy(os.path.join(src, "data.main"), tmp_path / "data.main")
    r = subprocess.run([FLUAM_REF, "data.main"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert "END" in r.stdout, r.stdout[-1000:]
    for ext in (".fluidFinalConfiguration", ".temperature", ".seed"):
        assert open(tmp_path / ("out" + ext)).read() == open(os.path.join(src, "out" + ext)).read()
