"""Soft repulsion through the Verlet pair list (the default for soft pairs on
the 3-D Stokes schemes) against the cell-list force kernel
(FLUAMSL_VERLET=0): the list holds every pair within rc + skin at its
reference positions and is rebuilt once a particle has moved more than
skin / 2, after positions are set from the host, and when a component entry
point asks for the lists, so the pair set equals the cell-list one; only the
order of the force sums differs (FP64 rounding)."""
import os

import numpy as np
import pytest

from helpers import chains, uniform_positions

pytestmark = pytest.mark.gpu


def _make(fsl, q, verlet, kT=1.0, dt=0.05, kernel=4, bonds=None, m=(32, 32, 32), L=32.0, scheme=0):
    cfg = fsl.make_config(m, (L,) * 3, eta=1.0, kT=kT, dt=dt, cutoff=1.5, kernel=kernel,
                          pair=fsl.PAIR_SOFT, soft_epsilon=1.0, seed=9, scheme=scheme)
    old = os.environ.get("FLUAMSL_VERLET")
    os.environ["FLUAMSL_VERLET"] = "1" if verlet else "0"
    try:
        s = fsl.StokesLimit(cfg, q)
    finally:
        if old is None:
            del os.environ["FLUAMSL_VERLET"]
        else:
            os.environ["FLUAMSL_VERLET"] = old
    if bonds is not None:
        s.load_bonds(*bonds)
    return s


def _pair(fsl, q, **kw):
    return _make(fsl, q, False, **kw), _make(fsl, q, True, **kw)


@pytest.mark.parametrize("scheme", [0, 1])
def test_verlet_follows_cell_list(fsl, scheme):
    """Fast diffusion (a particle crosses skin / 2 every few steps, so the
    list is rebuilt many times) with bonded chains and dense contacts."""
    q, bi, bj = chains(24, 16, (32.0,) * 3, 5)
    bonds = (bi, bj, np.full(len(bi), 10.0), np.ones(len(bi)))
    a, b = _pair(fsl, q, bonds=bonds, scheme=scheme)
    with a, b:
        for _ in range(6):
            a.step(5)
            b.step(5)
            qa, qb = a.positions(), b.positions()
            span = np.abs(qa - q).max()
            assert span > 0.2  # well past skin / 2 = 0.1875: rebuilt
            assert np.abs(qa - qb).max() <= 1e-9 * span
            Fa, Fb = a.forces(), b.forces()
            assert np.abs(Fa - Fb).max() <= 1e-9 * max(1.0, np.abs(Fa).max())
        assert a.status()["error_bits"] == 0 and b.status()["error_bits"] == 0


def test_verlet_after_set_positions_and_entry_points(fsl):
    q = uniform_positions(400, (32.0,) * 3, 3)
    a, b = _pair(fsl, q, kT=0.01, dt=0.01)
    with a, b:
        a.step(3)
        b.step(3)
        # a new configuration from the host: the list must be rebuilt
        q2 = uniform_positions(400, (32.0,) * 3, 4)
        a.set_positions(q2)
        b.set_positions(q2)
        a.step(2)
        b.step(2)
        np.testing.assert_allclose(b.positions(), a.positions(), rtol=0, atol=1e-12)
        # the component entry point on the current positions
        Fa, Fb = a.compute_forces(), b.compute_forces()
        np.testing.assert_allclose(Fb, Fa, rtol=0, atol=1e-12 * max(1.0, np.abs(Fa).max()))
        b.step(1)
        a.step(1)
        np.testing.assert_allclose(b.positions(), a.positions(), rtol=0, atol=1e-12)


def test_verlet_overflow_falls_back_to_cells(fsl):
    """More than 64 neighbours within rc + skin (a dense random box, as the
    served workload draws): the instance switches to the cell-list pair
    forces and follows the cell-list kernel."""
    q = uniform_positions(4000, (10.0,) * 3, 2)
    kw = dict(kT=0.01, dt=0.01, kernel=3, m=(16, 16, 16), L=10.0)
    a, b = _pair(fsl, q, **kw)
    with a, b:
        for _ in range(3):
            a.step(2)
            b.step(2)
            assert a.status()["error_bits"] == 0 and b.status()["error_bits"] == 0
            qa = a.positions()
            np.testing.assert_allclose(b.positions(), qa, rtol=0, atol=1e-12 * max(1.0, np.abs(qa).max()))
            Fa = a.forces()
            np.testing.assert_allclose(b.forces(), Fa, rtol=0, atol=1e-11 * max(1.0, np.abs(Fa).max()))


def test_list_barrier_give_up_is_reported_and_recovers(fsl, monkeypatch):
    """The single-launch list build's grid barrier waits with a bound.  With
    the bound at zero (FLUAMSL_COOP_SPIN_LIMIT=0, read when the step is
    enqueued) every wait gives up at once: the build stops in every block,
    the instance reports FSL_ERRBIT_GRID through fsl_sync (FSL_E_KERNEL), and
    after fsl_clear_errors the same instance steps to the same bits as a
    fresh one."""
    L = (32.0,) * 3
    q = uniform_positions(256, L, 41)

    def make():
        cfg = fsl.make_config((32, 32, 32), L, kT=0.01, dt=0.01, cutoff=1.5, kernel=3,
                              pair=fsl.PAIR_SOFT, seed=5)
        g = fsl.StokesLimit(cfg, q)
        g.set_graph(False)
        return g

    ref = make()
    ref.step(1)
    ref.sync()
    q1 = ref.positions()
    ref.close()

    g = make()
    monkeypatch.setenv("FLUAMSL_COOP_SPIN_LIMIT", "0")
    g.step(1)
    with pytest.raises(fsl._lib.FslError) as e:
        g.sync()
    assert e.value.code == -4
    assert g.status()["error_bits"] & 4
    monkeypatch.delenv("FLUAMSL_COOP_SPIN_LIMIT")
    g.clear_errors()
    g.set_positions(q)
    g.set_step(0)
    g.step(1)
    g.sync()
    assert g.status()["error_bits"] == 0
    np.testing.assert_array_equal(g.positions(), q1)
    g.close()
