"""FP64 observables accumulated on the device (fsl_config.observables = 1):
mean-square displacement from the reference positions, centre-of-mass
displacement, total particle force and fluid momentum, and their sums over
the steps.  The reference computes none of these on the Stokes path; the
check is against the same sums taken in numpy (FP64) over the instance's own
positions, forces and velocity field read back after every step.
"""
import numpy as np
import pytest

from helpers import chains, uniform_positions

pytestmark = pytest.mark.gpu


def _cfg(fsl, m=(32, 32, 32), L=32.0, kernel=3, precision=0, scheme=0, seed=3, observables=1):
    return fsl.make_config(m, (L,) * 3, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5, kernel=kernel,
                           pair=fsl.PAIR_SOFT, soft_epsilon=1.0, seed=seed, scheme=scheme,
                           precision=precision, observables=observables)


def _expected(q, q0, F, v, dV):
    d = q - q0
    return dict(msd=float(np.mean(np.sum(d * d, axis=0))), displacement=d.mean(axis=1),
                force=F.sum(axis=1), momentum=v.reshape(3, -1).sum(axis=1) * dV)


@pytest.mark.parametrize("precision,kernel,scheme", [(0, 3, 0), (0, 4, 1), (2, 3, 0)])
def test_observables_match_host_sums(fsl, precision, kernel, scheme):
    q0 = uniform_positions(300, (32.0,) * 3, 5)
    with fsl.StokesLimit(_cfg(fsl, kernel=kernel, precision=precision, scheme=scheme), q0) as s:
        msd_sum, mom_sum = 0.0, np.zeros(3)
        for n in range(1, 6):
            s.step(1)
            q, F, v = s.positions(), s.forces(), s.velocity64()
            e = _expected(q, q0, F, v, 1.0)
            o = s.observables()
            msd_sum += e["msd"]
            mom_sum += e["momentum"]
            assert o["steps"] == n
            assert o["msd"] == pytest.approx(e["msd"], rel=1e-12)
            assert o["msd_sum"] == pytest.approx(msd_sum, rel=1e-12)
            np.testing.assert_allclose(o["displacement"], e["displacement"], rtol=0,
                                       atol=1e-13 * max(1.0, np.abs(q - q0).max()))
            np.testing.assert_allclose(o["force"], e["force"], rtol=0, atol=1e-12 * np.abs(F).sum())
            scale = np.abs(v).sum()
            np.testing.assert_allclose(o["momentum"], e["momentum"], rtol=0, atol=1e-12 * scale)
            np.testing.assert_allclose(o["momentum_sum"], mom_sum, rtol=0, atol=1e-11 * scale)
            # pair forces are equal and opposite; the k = 0 mode of the solve is zero
            assert np.abs(o["force"]).max() <= 1e-10 * np.abs(F).sum()
            assert np.abs(o["momentum"]).max() <= 1e-5 * scale


def test_observables_bitwise_repeatable_and_batched(fsl):
    q0, bi, bj = chains(12, 16, (32.0,) * 3, 7)
    k, r0 = np.full(len(bi), 10.0), np.ones(len(bi))
    runs = []
    for _ in range(2):
        with fsl.StokesLimit(_cfg(fsl, kernel=4), q0) as s:
            s.load_bonds(bi, bj, k, r0)
            s.step(8)
            runs.append(s.observables())
    assert runs[0] == runs[1]
    other = uniform_positions(100, (24.0,) * 3, 9)
    cfgs = [_cfg(fsl, kernel=4), _cfg(fsl, m=(24, 24, 24), L=24.0, seed=4), _cfg(fsl, kernel=4)]
    with fsl.Batch(cfgs, [q0, other, q0]) as b:
        b.load_bonds(0, bi, bj, k, r0)
        b.load_bonds(2, bi, bj, k, r0)
        b.step(8)
        assert b.observables(0) == runs[0]
        assert b.observables(2) == runs[0]
        assert b.observables(1)["steps"] == 8


def test_reset_observables(fsl):
    q0 = uniform_positions(200, (32.0,) * 3, 8)
    with fsl.StokesLimit(_cfg(fsl), q0) as s:
        s.step(3)
        s.reset_observables()
        o = s.observables()
        assert o["steps"] == 0 and o["msd"] == 0.0 and o["msd_sum"] == 0.0
        q1 = s.positions()
        s.step(1)
        d = s.positions() - q1
        assert s.observables()["msd"] == pytest.approx(float(np.mean(np.sum(d * d, axis=0))), rel=1e-12)


def test_observables_off_and_refused(fsl):
    from fluam_b200._lib import FslError
    q0 = uniform_positions(50, (32.0,) * 3, 8)
    with fsl.StokesLimit(_cfg(fsl, observables=0), q0) as s:
        s.step(1)
        with pytest.raises(FslError):
            s.observables()
        # no extra launch when off
        n_off = s.status()["launches_per_step"]
    with fsl.StokesLimit(_cfg(fsl), q0) as s:
        s.step(1)
        assert s.status()["launches_per_step"] == n_off + 1
    q2 = uniform_positions(50, (32.0, 32.0, 1.0), 8)
    with pytest.raises(FslError):
        fsl.StokesLimit(fsl.make_config((32, 32, 1), (32.0, 32.0, 1.0), kT=0.01, dt=0.01,
                                        scheme=fsl.SCHEME_QUASI2D, observables=1), q2)


def test_data_main_observables_file(tmp_path, fsl):
    """observables 1 in data.main: <out>.observables, one line per sample,
    whose msd matches the positions in <out>.particles."""
    from golden_cases import read_particles, simple_cubic
    from test_dropin_gpu import run_fluam
    out = tmp_path / "run"
    text = f"""stokesLimit
particles 1
numberparticles 64
cutoff 1.5
pairPotential soft
shearviscosity 1
temperature 0.05
cells 16 16 16
celldimension 16 16 16
seed 3
numsteps 6
samplefreq 3
dt 0.01
observables 1
outputname {out}
"""
    run_fluam(tmp_path, text)
    rows = [r.split() for r in (tmp_path / "run.observables").read_text().strip().split("\n")]
    assert rows[0][0] == "#" and len(rows) == 3
    vals = np.array(rows[1:], dtype=float)
    assert vals.shape == (2, 12)
    _, pos = read_particles(tmp_path / "run.particles")
    q0 = simple_cubic(64, 16.0, 16.0, 16.0)
    for row in vals:
        d = pos[row[0]] - q0
        assert row[1] == pytest.approx(float(np.mean(np.sum(d * d, axis=0))), rel=1e-9)
