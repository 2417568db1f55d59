"""The tiled spread + W build of the fixed-point form against the global-atomic
spread and the separate W build: every node's fixed-point sum is the same
integer and W is built with the same arithmetic, so positions, forces and
the velocity field agree bit for bit.  FLUAMSL_TILED_SPREAD=1 selects the
tiled path when an instance is created (the global-atomic path is the
default)."""
import os

import numpy as np
import pytest

from helpers import chains, uniform_positions

pytestmark = pytest.mark.gpu

CASES = {
    "3pt_soft_32": dict(m=(32, 32, 32), L=(32.0,) * 3, n=300, kernel=3, pair="soft"),
    "4pt_chains_32": dict(m=(32, 32, 32), L=(32.0,) * 3, n=None, kernel=4, pair="soft"),
    # partial tiles in every direction, LJ table, extraMobility
    "4pt_lj_ragged": dict(m=(40, 24, 20), L=(40.0, 24.0, 20.0), n=200, kernel=4, pair="lj", extra=0.3),
    # mx not a multiple of 4: the scalar W build
    "3pt_odd_x": dict(m=(21, 18, 25), L=(21.0, 18.0, 25.0), n=150, kernel=3, pair="soft"),
    # neighbour ranges wrapping the whole grid; cells not a multiple of dx
    "4pt_small": dict(m=(16, 16, 16), L=(12.0, 12.0, 12.0), n=120, kernel=4, pair="soft"),
    "3pt_paper": dict(m=(24, 32, 16), L=(24.0, 32.0, 16.0), n=200, kernel=3, pair="soft", rfd="paper"),
    "4pt_first_order": dict(m=(32, 24, 24), L=(32.0, 24.0, 24.0), n=250, kernel=4, pair="soft",
                            scheme="first"),
}


def _run(fsl, c, tiled, steps=6):
    L = c["L"]
    if c["n"] is None:
        q, bi, bj = chains(16, 16, L, 3)
    elif c["pair"] == "lj":
        # a jittered lattice of spacing 3: no overlaps for the LJ table
        g = [np.arange(int(x // 3)) * 3.0 - x / 2 + 1.5 for x in L]
        q = np.stack(np.meshgrid(*g, indexing="ij")).reshape(3, -1)[:, :c["n"]]
        q = q + 0.2 * (uniform_positions(q.shape[1], (1.0,) * 3, 5))
        bi = None
    else:
        q, bi = uniform_positions(c["n"], L, 17), None
    cfg = fsl.make_config(c["m"], L, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5, kernel=c["kernel"],
                          pair={"soft": fsl.PAIR_SOFT, "lj": fsl.PAIR_TABLE_LJ}[c["pair"]],
                          soft_epsilon=1.0, extra_mobility=c.get("extra", 0.0),
                          rfd=fsl.RFD_PAPER if c.get("rfd") == "paper" else fsl.RFD_REFERENCE,
                          scheme=fsl.SCHEME_FIRST_ORDER if c.get("scheme") == "first" else 0,
                          seed=21)
    old = os.environ.get("FLUAMSL_TILED_SPREAD"), os.environ.get("FLUAMSL_VERLET")
    os.environ["FLUAMSL_TILED_SPREAD"] = "1" if tiled else "0"
    os.environ["FLUAMSL_VERLET"] = "0"  # the tiles read the cell lists of every step
    try:
        with fsl.StokesLimit(cfg, q) as s:
            if bi is not None:
                s.load_bonds(bi, bj, np.full(len(bi), 10.0), np.ones(len(bi)))
            s.step(steps)
            st = s.status()
            assert st["error_bits"] == 0
            out = s.positions(), s.forces(), s.velocity()
            # the stages of one more (profiled) step, after the state was read
            s.profile(True)
            s.step(1)
            s.sync()
            stages = set(s.profile_read())
            s.profile(False)
            return out + (stages,)
    finally:
        for key, val in zip(("FLUAMSL_TILED_SPREAD", "FLUAMSL_VERLET"), old):
            if val is None:
                del os.environ[key]
            else:
                os.environ[key] = val


@pytest.mark.parametrize("name", sorted(CASES))
def test_tiled_equals_atomic(fsl, name):
    q0, F0, v0, s0 = _run(fsl, CASES[name], False)
    q1, F1, v1, s1 = _run(fsl, CASES[name], True)
    # the tiled path ran: its spread writes W, the other spreads into the field
    assert any(k.startswith("spread_w") for k in s1) and not any(k.startswith("spread_w") for k in s0)
    np.testing.assert_array_equal(q1, q0)
    np.testing.assert_array_equal(F1, F0)
    np.testing.assert_array_equal(v1, v0)
