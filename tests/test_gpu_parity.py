"""Parity of the CUDA path (through the C ABI) with the FP64 CPU oracle.

Integer work (cell lists, stencil choice) must be bit-exact; floating-point
results must agree within the stated FP32 tolerance TOL = 1e-5 relative
(max |gpu - oracle| / max |oracle|) per step, from the same state.
"""
import numpy as np
import pytest

from helpers import chains, rel_inf, uniform_positions

pytestmark = pytest.mark.gpu

TOL = 1e-5


def make_pair(fsl, oracle, m, L, q, *, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5, kernel=3,
              pair="soft", eps=1.0, rfd="reference", nonbonded=1, extra=0.0, seed=7,
              scheme="midpoint"):
    pg = {"none": fsl.PAIR_NONE, "lj": fsl.PAIR_TABLE_LJ, "soft": fsl.PAIR_SOFT}[pair]
    po = {"none": oracle.PAIR_NONE, "lj": oracle.PAIR_TABLE_LJ, "soft": oracle.PAIR_SOFT}[pair]
    rg = fsl.RFD_REFERENCE if rfd == "reference" else fsl.RFD_PAPER
    ro = oracle.RFD_REFERENCE if rfd == "reference" else oracle.RFD_PAPER
    cfg = fsl.make_config(m, L, eta=eta, kT=kT, dt=dt, cutoff=cutoff, kernel=kernel, pair=pg,
                          soft_epsilon=eps, rfd=rg, nonbonded=nonbonded, extra_mobility=extra,
                          seed=seed,
                          scheme=fsl.SCHEME_FIRST_ORDER if scheme == "first" else fsl.SCHEME_MIDPOINT)
    g = fsl.StokesLimit(cfg, q)
    o = oracle.Oracle(m[0], m[1], m[2], L[0], L[1], L[2], q, eta=eta, kT=kT, dt=dt, cutoff=cutoff,
                      kernel=kernel, pair=po, soft_epsilon=eps, rfd=ro, nonbonded=nonbonded,
                      extra_mobility=extra, seed=seed,
                      scheme=oracle.SCHEME_FIRST_ORDER if scheme == "first" else oracle.SCHEME_MIDPOINT)
    return g, o


def test_noise_matches_oracle(fsl, oracle):
    q = uniform_positions(10, (8, 8, 8), 1)
    g, o = make_pair(fsl, oracle, (8, 8, 8), (8.0, 8.0, 8.0), q, seed=99)
    for t, first, n in [(0, 0, 20000), (5, 12345, 1001), (2 ** 33 + 1, 7, 4096)]:
        a = g.noise(t, first, n)
        b = oracle.noise(99, t, first, n)
        assert np.abs(a - b).max() < 2e-5
    g.close()


@pytest.mark.parametrize("case", ["uniform", "unwrapped", "boundaries", "dense"])
def test_cell_list_bit_exact(fsl, oracle, case):
    L = (20.0, 16.0, 24.0)
    m = (20, 16, 24)
    if case == "uniform":
        q = uniform_positions(700, L, 3)
    elif case == "unwrapped":
        q = uniform_positions(700, L, 4) + np.array([[41.0], [-33.0], [97.0]])
    elif case == "boundaries":
        # on cell faces and on the box faces, both signs
        h = np.array([20.0 / 13, 16.0 / 10, 24.0 / 16]).reshape(3, 1)
        k = np.random.default_rng(5).integers(-8, 9, (3, 600))
        q = k * h
        q[:, :6] = np.array([[10.0, -10.0, 0.0, 10.0, -10.0, 20.0],
                             [8.0, -8.0, 0.0, -8.0, 8.0, 16.0],
                             [12.0, -12.0, 0.0, 12.0, 12.0, -24.0]])
    else:
        q = uniform_positions(3000, L, 6) * 0.3
    g, o = make_pair(fsl, oracle, m, L, q)
    assert g.neighbor_grid() == o.neighbor_grid()[0]
    c1, s1, p1 = g.cell_list()
    c2, s2, p2 = o.cell_list(q)
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(p1, p2)
    g.close()


@pytest.mark.parametrize("pair", ["soft", "lj"])
def test_pair_forces(fsl, oracle, pair):
    L = (16.0, 16.0, 16.0)
    q = uniform_positions(1500, L, 8)  # overlaps included: forces only, no spreading
    cutoff = 1.5 if pair == "soft" else 2 ** (1 / 6) * 1.0  # sigma = 2 dx with dx = 0.5
    g, o = make_pair(fsl, oracle, (32, 32, 32), L, q, pair=pair, cutoff=cutoff, kT=0.3)
    Fg = g.compute_forces()
    Fo = o.compute_forces(q)
    assert rel_inf(Fg, Fo) < 1e-12
    g.close()


def test_bonded_forces(fsl, oracle):
    L = (24.0, 24.0, 24.0)
    q, bi, bj = chains(20, 16, L, 10)
    n = q.shape[1]
    g, o = make_pair(fsl, oracle, (24, 24, 24), L, q, pair="soft")
    k = np.full(len(bi), 10.0)
    r0 = np.where(np.arange(len(bi)) % 3 == 0, 0.0, 1.0)
    fi = np.array([0, 5, 5], np.int32)
    fk = np.array([1.0, 2.0, 3.0])
    fr0 = np.array([0.0, 0.5, 0.0])
    fxyz = np.array([[0.0, 0.0, 0.0], [1.0, 2.0, 3.0], [-4.0, 0.5, 2.0]])
    g.load_bonds(bi, bj, k, r0, fi, fk, fr0, fxyz)
    o.set_bonds(bi, bj, k, r0, fi, fk, fr0, fxyz)
    assert rel_inf(g.compute_forces(), o.compute_forces(q)) < 1e-12
    with pytest.raises(fsl._lib.FslError):
        g.load_bonds([0], [n], [1.0], [1.0])
    g.close()


def test_bonded_forces_directed(fsl, oracle):
    """Directed entries (the old bond-file format): each acts on its first
    particle only; the same entries listed from both ends equal the bonds."""
    L = (24.0, 24.0, 24.0)
    q, bi, bj = chains(10, 8, L, 14)
    g, o = make_pair(fsl, oracle, (24, 24, 24), L, q, pair="soft")
    k = 4.0 + np.arange(len(bi)) % 3
    r0 = np.where(np.arange(len(bi)) % 2 == 0, 1.0, 0.5)
    # both ends of every bond, sorted by the first index, plus two one-sided springs
    ei = np.concatenate([bi, bj, [3, 40]]).astype(np.int32)
    ej = np.concatenate([bj, bi, [70, 1]]).astype(np.int32)
    ek = np.concatenate([k, k, [2.0, 5.0]])
    er = np.concatenate([r0, r0, [1.5, 0.0]])
    order = np.argsort(ei, kind="stable")
    ei, ej, ek, er = ei[order], ej[order], ek[order], er[order]
    g.load_bonds(ei, ej, ek, er, directed=True)
    o.set_bonds(ei, ej, ek, er, directed=True)
    Fd = g.compute_forces()
    assert rel_inf(Fd, o.compute_forces(q)) < 1e-12
    # without the one-sided springs the directed entries are the bonds
    keep = ~(((ei == 3) & (ej == 70)) | ((ei == 40) & (ej == 1)))
    g.load_bonds(ei[keep], ej[keep], ek[keep], er[keep], directed=True)
    Fsym = g.compute_forces()
    g.load_bonds(bi, bj, k, r0)
    assert rel_inf(Fsym, g.compute_forces()) < 1e-12
    g.close()


@pytest.mark.parametrize("kernel", [3, 4])
def test_spread(fsl, oracle, kernel):
    L = (16.0, 12.0, 20.0)
    m = (32, 24, 40)
    q = uniform_positions(400, L, 12) * 1.3
    g, o = make_pair(fsl, oracle, m, L, q, kernel=kernel)
    F = np.random.default_rng(2).standard_normal((3, 400))
    assert rel_inf(g.spread(F), o.spread(q, F)) < TOL
    g.close()


@pytest.mark.parametrize("m", [(32, 32, 32), (16, 24, 40), (22, 18, 20), (56, 8, 12), (12, 10, 14),
                               (16, 16, 16), (24, 24, 24), (48, 48, 48), (64, 64, 64), (96, 96, 96),
                               (128, 128, 128), (32, 32, 256), (64, 64, 24),
                               # register passes with radix 5, 7, 11 and T = 6
                               (40, 40, 40), (56, 56, 56), (72, 72, 72), (80, 80, 80), (88, 88, 88),
                               (40, 40, 88), (88, 88, 56)])
def test_solve(fsl, oracle, m):
    L = tuple(float(x) * 0.75 for x in m)
    q = uniform_positions(4, L, 1)
    g, o = make_pair(fsl, oracle, m, L, q, eta=1.3)
    W = np.random.default_rng(5).standard_normal((3, m[2], m[1], m[0]))
    assert rel_inf(g.solve(W), o.solve(W)) < TOL
    g.close()


@pytest.mark.parametrize("kernel", [3, 4])
def test_interpolate(fsl, oracle, kernel):
    L = (16.0, 12.0, 20.0)
    m = (32, 24, 40)
    q = uniform_positions(400, L, 13) * 1.5
    g, o = make_pair(fsl, oracle, m, L, q, kernel=kernel)
    v = np.random.default_rng(6).standard_normal((3, m[2], m[1], m[0]))
    assert rel_inf(g.interpolate(v), o.interp(q, v)) < TOL
    g.close()


STEP_CASES = {
    "c1_3pt_soft": dict(m=(32, 32, 32), L=(32.0,) * 3, n=256, kernel=3, pair="soft"),
    "3pt_lj": dict(m=(32, 32, 32), L=(16.0,) * 3, n=300, kernel=3, pair="lj", cutoff=2 ** (1 / 6),
                   kT=0.05),
    "4pt_soft_chains": dict(m=(32, 32, 32), L=(32.0,) * 3, n=None, kernel=4, pair="soft", dt=0.005),
    "3pt_paper_rfd": dict(m=(24, 24, 24), L=(24.0,) * 3, n=200, kernel=3, pair="soft", rfd="paper"),
    "4pt_paper_rfd_extra": dict(m=(20, 24, 28), L=(20.0, 24.0, 28.0), n=150, kernel=4, pair="soft",
                                rfd="paper", extra=0.3),
    "3pt_no_pairs": dict(m=(16, 16, 16), L=(16.0,) * 3, n=64, kernel=3, pair="none"),
    # the first-order integrator (keyword stokesLimitFirstOrder)
    "first_3pt_soft": dict(m=(32, 32, 32), L=(32.0,) * 3, n=256, kernel=3, pair="soft",
                           scheme="first"),
    "first_3pt_lj": dict(m=(32, 32, 32), L=(16.0,) * 3, n=300, kernel=3, pair="lj",
                         cutoff=2 ** (1 / 6), kT=0.05, scheme="first"),
    "first_4pt_chains_extra": dict(m=(32, 32, 32), L=(32.0,) * 3, n=None, kernel=4, pair="soft",
                                   dt=0.005, extra=0.3, scheme="first"),
    "first_4pt_paper_rfd": dict(m=(20, 24, 28), L=(20.0, 24.0, 28.0), n=150, kernel=4,
                                pair="soft", rfd="paper", scheme="first"),
}


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_step_teacher_forced(fsl, oracle, name):
    """Each step from the oracle's state: displacement, F^{n+1/2} and v agree."""
    c = dict(STEP_CASES[name])
    m, L, n = c.pop("m"), c.pop("L"), c.pop("n")
    bonds = None
    if n is None:
        q, bi, bj = chains(16, 16, L, 3)
        bonds = (bi, bj, np.full(len(bi), 10.0), np.ones(len(bi)))
    elif c.get("pair") == "lj":
        # LJ needs a configuration without overlaps: a jittered lattice just
        # inside the cutoff (sigma = 2 dx = 1)
        g3 = np.stack(np.meshgrid(np.arange(7), np.arange(7), np.arange(6), indexing="ij"))
        q = (g3.reshape(3, -1) * 1.05 - 3.0)
        q = q + np.random.default_rng(17).uniform(-0.04, 0.04, q.shape)
    else:
        q = uniform_positions(n, L, 17)
    g, o = make_pair(fsl, oracle, m, L, q, **c)
    if bonds:
        g.load_bonds(*bonds)
        o.set_bonds(*bonds)
    g.set_graph(False)
    for t in range(3):
        q0 = o.positions()
        g.set_positions(q0)
        g.set_step(t)
        o.t = t
        g.step(1)
        o.step(1)
        g.sync()
        dq_g = g.positions() - q0
        dq_o = o.positions() - q0
        assert rel_inf(dq_g, dq_o) < TOL, (t, rel_inf(dq_g, dq_o))
        assert rel_inf(g.forces(), o.forces()) < TOL
        assert rel_inf(g.velocity(), o.velocity()) < TOL
    g.close()


def test_free_run_tracks_oracle(fsl, oracle):
    L = (32.0,) * 3
    q = uniform_positions(256, L, 23)
    g, o = make_pair(fsl, oracle, (32, 32, 32), L, q)
    g.step(10)
    o.step(10)
    g.sync()
    assert rel_inf(g.positions() - q, o.positions() - q) < 1e-4


def test_bit_reproducible_and_graph_equivalent(fsl, oracle):
    L = (32.0,) * 3
    q, bi, bj = chains(16, 16, L, 5)
    runs = []
    for graph in (True, True, False):
        cfg = fsl.make_config((32, 32, 32), L, kT=0.01, dt=0.005, cutoff=1.5, kernel=4,
                              pair=fsl.PAIR_SOFT, seed=3)
        g = fsl.StokesLimit(cfg, q)
        g.load_bonds(bi, bj, np.full(len(bi), 10.0), np.ones(len(bi)))
        g.set_graph(graph)
        g.step(6)
        g.sync()
        runs.append((g.positions(), g.forces(), g.velocity(), g.status()))
        g.close()
    for r in runs[1:]:
        np.testing.assert_array_equal(r[0], runs[0][0])
        np.testing.assert_array_equal(r[1], runs[0][1])
        np.testing.assert_array_equal(r[2], runs[0][2])
    assert runs[0][3]["graph"] and not runs[2][3]["graph"]
    assert runs[0][3]["step"] == 6


def test_fixed_point_saturation_is_reported(fsl, oracle):
    """An out-of-range spread value raises the error word, not a fault."""
    L = (16.0,) * 3
    q = uniform_positions(8, L, 2)
    cfg = fsl.make_config((16, 16, 16), L, kT=0.0, dt=0.01, cutoff=1.5, pair=fsl.PAIR_NONE)
    g = fsl.StokesLimit(cfg, q)
    g.load_bonds([0], [1], [1e30], [0.0])
    g.step(1)
    with pytest.raises(fsl._lib.FslError) as e:
        g.sync()
    assert e.value.code == -4
    assert g.status()["error_bits"] & 1
    g.clear_errors()
    assert g.status()["error_bits"] == 0
    g.close()
