"""The three precision forms of the fluid side against the FP64 oracle.

(a) FIXED64: FP32 fields, 64-bit fixed-point spreading (the default);
(b) FLOAT_ATOMIC: FP32 fields, FP32 atomic spreading;
(c) FP64: everything in double on the GPU.

Each step starts from the oracle's state (teacher forcing) and the
displacement, the forces and the fluid velocity are compared with the
oracle's.  Stated tolerances (max |gpu - oracle| / max |oracle|): FP32 forms
1e-5, the FP64 form 1e-10.
"""
import numpy as np
import pytest

from helpers import chains, rel_inf, uniform_positions

pytestmark = pytest.mark.gpu

TOL = {0: 1e-5, 1: 1e-5, 2: 1e-10}

CASES = {
    "3pt_soft": dict(m=(32, 32, 32), L=(32.0,) * 3, n=256, kernel=3, pair="soft", dt=0.01),
    "4pt_chains_extra": dict(m=(32, 32, 32), L=(32.0,) * 3, n=None, kernel=4, pair="soft",
                             dt=0.005, extra=0.3),
    # non-power-of-two lines (radices 5 and 7 and 3) and the paper RFD
    "3pt_ragged_paper": dict(m=(20, 24, 28), L=(20.0, 24.0, 28.0), n=150, kernel=3,
                             pair="soft", rfd="paper", dt=0.01),
    "first_order_4pt": dict(m=(24, 24, 24), L=(24.0,) * 3, n=200, kernel=4, pair="soft",
                            dt=0.01, scheme="first"),
}


def make(fsl, oracle, prec, m, L, n, kernel, pair, dt, extra=0.0, rfd="reference",
         scheme="midpoint", seed=11):
    if n is None:
        q, bi, bj = chains(16, 16, L, 3)
        bonds = (bi, bj, np.full(len(bi), 10.0), np.ones(len(bi)))
    else:
        q = uniform_positions(n, L, 29)
        bonds = None
    pg = {"soft": fsl.PAIR_SOFT, "none": fsl.PAIR_NONE}[pair]
    po = {"soft": oracle.PAIR_SOFT, "none": oracle.PAIR_NONE}[pair]
    first = scheme == "first"
    cfg = fsl.make_config(m, L, eta=1.0, kT=0.01, dt=dt, cutoff=1.5, kernel=kernel, pair=pg,
                          rfd=fsl.RFD_PAPER if rfd == "paper" else fsl.RFD_REFERENCE,
                          extra_mobility=extra, seed=seed,
                          scheme=fsl.SCHEME_FIRST_ORDER if first else fsl.SCHEME_MIDPOINT,
                          precision=prec)
    g = fsl.StokesLimit(cfg, q)
    o = oracle.Oracle(m[0], m[1], m[2], L[0], L[1], L[2], q, eta=1.0, kT=0.01, dt=dt,
                      cutoff=1.5, kernel=kernel, pair=po,
                      rfd=oracle.RFD_PAPER if rfd == "paper" else oracle.RFD_REFERENCE,
                      extra_mobility=extra, seed=seed,
                      scheme=oracle.SCHEME_FIRST_ORDER if first else oracle.SCHEME_MIDPOINT)
    if bonds:
        g.load_bonds(*bonds)
        o.set_bonds(*bonds)
    return g, o


@pytest.mark.parametrize("prec", [0, 1, 2], ids=["fixed64", "float_atomic", "fp64"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_teacher_forced_against_oracle(fsl, oracle, name, prec):
    g, o = make(fsl, oracle, prec, **CASES[name])
    g.set_graph(False)
    tol = TOL[prec]
    for t in range(3):
        q0 = o.positions()
        g.set_positions(q0)
        g.set_step(t)
        o.t = t
        g.step(1)
        o.step(1)
        g.sync()
        e_q = rel_inf(g.positions() - q0, o.positions() - q0)
        e_f = rel_inf(g.forces(), o.forces())
        e_v = rel_inf(g.velocity64(), o.velocity())
        assert e_q < tol and e_f < tol and e_v < tol, (t, e_q, e_f, e_v)
    g.close()


def test_fp64_form_is_closer_than_fp32(fsl, oracle):
    """Free run of 20 steps: the FP64 form stays orders of magnitude closer
    to the oracle than the fixed-point FP32 form."""
    errs = {}
    for prec in (0, 2):
        g, o = make(fsl, oracle, prec, **CASES["3pt_soft"])
        q0 = o.positions()
        g.step(20)
        o.step(20)
        g.sync()
        errs[prec] = rel_inf(g.positions() - q0, o.positions() - q0)
        g.close()
    assert errs[2] < 1e-9 and errs[2] < 1e-3 * errs[0], errs


@pytest.mark.parametrize("prec", [0, 2], ids=["fixed64", "fp64"])
def test_graph_replay_is_bit_identical(fsl, oracle, prec):
    """Run to run and graph vs eager: bit-identical for the fixed-point form;
    the FP64 form's atomics make it order dependent, so it is compared within
    its tolerance."""
    runs = []
    for graph in (True, True, False):
        g, _ = make(fsl, oracle, prec, **CASES["4pt_chains_extra"])
        g.set_graph(graph)
        g.step(8)
        g.sync()
        runs.append(g.positions())
        g.close()
    q0 = runs[0]
    if prec == 0:
        assert all(np.array_equal(r, q0) for r in runs[1:])
    else:
        assert all(np.abs(r - q0).max() < 1e-10 for r in runs[1:])


def test_batch_of_mixed_forms_equals_alone(fsl, oracle):
    """Instances of the three forms in one batch (three size classes): the
    fixed-point one gives the bits it gives alone, the atomic-order dependent
    ones agree within their tolerances."""
    c = CASES["3pt_soft"]
    q = uniform_positions(c["n"], c["L"], 29)
    cfgs = [fsl.make_config(c["m"], c["L"], eta=1.0, kT=0.01, dt=0.01, cutoff=1.5, kernel=3,
                            pair=fsl.PAIR_SOFT, seed=5 + p, precision=p) for p in (0, 1, 2)]
    alone = []
    for cfg in cfgs:
        g = fsl.StokesLimit(cfg, q)
        g.step(5)
        g.sync()
        alone.append(g.positions())
        g.close()
    b = fsl.Batch(cfgs, [q, q, q])
    b.step(5)
    b.sync()
    assert np.array_equal(b.positions(0), alone[0])
    assert rel_inf(b.positions(1) - q, alone[1] - q) < 1e-4
    assert rel_inf(b.positions(2) - q, alone[2] - q) < 1e-10
    b.close()


def test_stage_entry_points_refuse_other_forms(fsl):
    import ctypes
    q = uniform_positions(16, (16.0,) * 3, 1)
    for prec in (1, 2):
        cfg = fsl.make_config((16, 16, 16), (16.0,) * 3, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5,
                              kernel=3, pair=fsl.PAIR_SOFT, seed=1, precision=prec)
        g = fsl.StokesLimit(cfg, q)
        W = np.zeros((3, 16, 16, 16))
        v = np.zeros_like(W)
        rc = g.L.fsl_solve(g.h, W.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert rc == -1  # FSL_E_ARG
        g.close()


def test_precision_study_small(tmp_path):
    """The study script end to end on a small case (64^3, 4,096 particles)."""
    import precision_study
    r = precision_study.main(["--cells", "64", "--np", "4096", "--steps", "6", "--oracle-steps", "1",
                              "--json", str(tmp_path / "s.json"), "--md", str(tmp_path / "s.md")])
    pin = r["oracle_pin"][0]
    assert pin["fp64"]["dq_rel_inf"] < 1e-10 and pin["fp64"]["v_rel_inf"] < 1e-10
    assert pin["fixed64"]["dq_rel_inf"] < 1e-5 and pin["float_atomic"]["dq_rel_inf"] < 1e-5
    assert r["per_step_vs_fp64_form"]["fixed64"]["dq_rel_inf_max"] < 1e-5
    assert r["reproducibility"]["fixed64"]["bit_identical"]
    assert (tmp_path / "s.md").read_text().startswith("# Precision study")
