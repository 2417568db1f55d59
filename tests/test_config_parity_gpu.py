"""Parity with the FP64 oracle on the benchmark configurations themselves.

* C2 (the headline workload, ``plain_128``): 128^3 cells, 65,536 particles
  as 4,096 bead-spring chains of 16 beads, 4-point kernel, soft repulsion
  through the Verlet list, dt 0.005.  Three steps, each started from the
  oracle's state, on the production path (CUDA graph, single-launch list
  build, autotuned transform schedule).
* C1: 32^3 cells, 256 uniform particles, 3-point kernel, soft repulsion,
  kT 0.01, dt 0.01, 100 steps.  Every step is started from the oracle's
  state and the displacement, the particle forces F^{n+1/2} and the fluid
  velocity field are compared at every step.

Tolerance as in test_gpu_parity.py: TOL = 1e-5 relative
(max |gpu - oracle| / max |oracle|) per step.
"""
import numpy as np
import pytest

from helpers import rel_inf, uniform_positions

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _oracle_for(oracle, w, q, seed):
    m, L = w["cells"], w["box"]
    return oracle.Oracle(m, m, m, L, L, L, q, eta=w["eta"], kT=w["kT"], dt=w["dt"], cutoff=w["rc"],
                         kernel=w["kernel"], pair=oracle.PAIR_SOFT, soft_epsilon=w["eps"], seed=seed)


def test_c2_plain_128_teacher_forced(fsl, oracle):
    from fluam_b200 import workloads
    seed = 1
    cfg, q, bonds = workloads.build("plain_128", seed=seed)
    w = workloads.WORKLOADS["plain_128"]
    assert q.shape == (3, 65536) and len(bonds[0]) == 4096 * 15
    g = fsl.StokesLimit(cfg, q)
    g.load_bonds(*bonds)
    o = _oracle_for(oracle, w, q, seed)
    o.set_bonds(*bonds)
    errs = []
    for t in range(3):
        q0 = o.positions()
        g.set_positions(q0)
        g.set_step(t)
        o.t = t
        g.step(1)
        o.step(1)
        g.sync()
        e = (rel_inf(g.positions() - q0, o.positions() - q0), rel_inf(g.forces(), o.forces()),
             rel_inf(g.velocity(), o.velocity()))
        errs.append(e)
        assert max(e) < TOL, (t, e)
    st = g.status()
    assert st["graph"] and st["error_bits"] == 0
    g.close()
    print("C2 per-step relative errors (displacement, force, velocity):", errs)


def test_c1_100_steps_every_step(fsl, oracle):
    n, m, L = 256, 32, 32.0
    q = uniform_positions(n, (L, L, L), 2024)
    cfg = fsl.make_config((m, m, m), (L, L, L), eta=1.0, kT=0.01, dt=0.01, cutoff=1.5, kernel=3,
                          pair=fsl.PAIR_SOFT, soft_epsilon=1.0, seed=31)
    g = fsl.StokesLimit(cfg, q)
    o = oracle.Oracle(m, m, m, L, L, L, q, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5, kernel=3,
                      pair=oracle.PAIR_SOFT, soft_epsilon=1.0, seed=31)
    worst = np.zeros(3)
    for t in range(100):
        q0 = o.positions()
        g.set_positions(q0)
        g.set_step(t)
        o.t = t
        g.step(1)
        o.step(1)
        g.sync()
        e = np.array([rel_inf(g.positions() - q0, o.positions() - q0), rel_inf(g.forces(), o.forces()),
                      rel_inf(g.velocity(), o.velocity())])
        assert e.max() < TOL, (t, e)
        worst = np.maximum(worst, e)
    # the trajectory moved: 100 steps of Brownian motion at kT 0.01
    assert np.abs(o.positions() - q).max() > 1e-3
    g.close()
    print("C1 worst per-step relative errors over 100 steps (displacement, force, velocity):", worst)
