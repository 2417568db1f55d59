"""Batched instances through the fsl_batch_* C ABI.

Every instance of a batch must give exactly (bit for bit) what the same
instance gives stepped alone through fsl_create/fsl_step: the kernels of a
batch are the single-instance kernels reading their instance from a table,
and nothing couples instances.  One batch instance is also checked against
the FP64 oracle with the free-run tolerance of the plain path (1e-4 relative
displacement error after 3 steps).
"""
import numpy as np
import pytest

from helpers import chains, rel_inf, uniform_positions

pytestmark = pytest.mark.gpu


def mixed_set(fsl, n=10, seed=3, edges=(16, 24, 32), np_max=400, kernels=(3, 4)):
    """Seeded instances of several size classes, one without particles."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        m = int(rng.choice(edges))
        npart = 0 if i == 3 else int(round(np.exp(rng.uniform(np.log(8), np.log(np_max)))))
        kernel = int(rng.choice(kernels))
        cfg = fsl.make_config((m, m, m), (float(m),) * 3, eta=float(rng.uniform(0.5, 2.0)), kT=0.01,
                              dt=0.01, cutoff=1.5, kernel=kernel, pair=fsl.PAIR_SOFT, seed=1000 + i)
        out.append((cfg, uniform_positions(npart, (m, m, m), 50 + i)))
    return out


def run_alone(fsl, cfg, q, steps, bonds=None):
    g = fsl.StokesLimit(cfg, q)
    if bonds is not None:
        g.load_bonds(*bonds)
    g.step(steps)
    g.sync()
    r = (g.positions(), g.forces(), g.status())
    g.close()
    return r


def test_batch_equals_alone(fsl):
    inst = mixed_set(fsl)
    b = fsl.Batch([c for c, _ in inst], [q for _, q in inst])
    info = b.info()
    assert info["n"] == len(inst)
    keys = {(c.mx, c.kernel) for c, _ in inst}
    assert info["classes"] == len(keys)
    b.step(4)
    b.sync()
    assert b.info()["graph"]
    for i, (cfg, q) in enumerate(inst):
        qa, Fa, sa = run_alone(fsl, cfg, q, 4)
        np.testing.assert_array_equal(b.positions(i), qa)
        np.testing.assert_array_equal(b.forces(i), Fa)
        st = b.status(i)
        assert st["step"] == 4 and st["error_bits"] == 0 and st["np"] == q.shape[1]
    b.close()


def test_batch_graph_equals_eager(fsl):
    inst = mixed_set(fsl, n=7, seed=11)
    res = []
    for graph in (True, False):
        b = fsl.Batch([c for c, _ in inst], [q for _, q in inst])
        b.set_graph(graph)
        b.step(3)
        b.sync()
        res.append(b.positions_packed())
        assert b.info()["graph"] == graph
        b.close()
    np.testing.assert_array_equal(res[0], res[1])


def test_batch_with_bonds_equals_alone(fsl):
    L = (24.0,) * 3
    q1, bi, bj = chains(8, 12, L, 4)
    bonds = (bi, bj, np.full(len(bi), 10.0), np.ones(len(bi)))
    cfg1 = fsl.make_config((24, 24, 24), L, kT=0.01, dt=0.005, cutoff=1.5, kernel=4,
                           pair=fsl.PAIR_SOFT, seed=21)
    cfg2 = fsl.make_config((24, 24, 24), L, eta=0.7, kT=0.01, dt=0.005, cutoff=1.5, kernel=4,
                           pair=fsl.PAIR_SOFT, seed=22)
    q2 = uniform_positions(200, L, 9)
    b = fsl.Batch([cfg1, cfg2], [q1, q2])
    b.load_bonds(0, *bonds)
    b.step(3)
    b.sync()
    qa, Fa, _ = run_alone(fsl, cfg1, q1, 3, bonds)
    qb, Fb, _ = run_alone(fsl, cfg2, q2, 3)
    np.testing.assert_array_equal(b.positions(0), qa)
    np.testing.assert_array_equal(b.forces(0), Fa)
    np.testing.assert_array_equal(b.positions(1), qb)
    b.close()


def test_packed_positions_round_trip(fsl):
    inst = mixed_set(fsl, n=6, seed=5)
    b = fsl.Batch([c for c, _ in inst], [q for _, q in inst])
    packed = b.positions_packed()
    for i, (_, q) in enumerate(inst):
        np.testing.assert_array_equal(b.unpack(packed, i), q)
    b.set_positions_packed(packed + 0.25)
    for i, (_, q) in enumerate(inst):
        np.testing.assert_array_equal(b.positions(i), q + 0.25)
    b.close()


def test_error_word_is_per_instance(fsl):
    """An instance that saturates the fixed-point field reports it; the
    others' results are unaffected."""
    L = (16.0,) * 3
    cfgs = [fsl.make_config((16, 16, 16), L, kT=0.01, dt=0.01, cutoff=1.5, pair=fsl.PAIR_SOFT,
                            seed=s) for s in (1, 2, 3)]
    qs = [uniform_positions(40, L, 30 + s) for s in range(3)]
    b = fsl.Batch(cfgs, qs)
    b.load_bonds(1, [0], [1], [1e30], [0.0])
    b.step(1)
    with pytest.raises(fsl._lib.FslError) as e:
        b.sync()
    assert e.value.code == -4 and "instance 1" in str(e.value)
    assert b.status(1)["error_bits"] & 1
    assert b.status(0)["error_bits"] == 0 and b.status(2)["error_bits"] == 0
    for i in (0, 2):
        qa, _, _ = run_alone(fsl, cfgs[i], qs[i], 1)
        np.testing.assert_array_equal(b.positions(i), qa)
    b.close()


def test_batch_instance_tracks_oracle(fsl, oracle):
    L = (32.0,) * 3
    q = uniform_positions(256, L, 23)
    cfg = fsl.make_config((32, 32, 32), L, kT=0.01, dt=0.01, cutoff=1.5, kernel=3,
                          pair=fsl.PAIR_SOFT, seed=7)
    other = fsl.make_config((16, 16, 16), (16.0,) * 3, kT=0.01, dt=0.01, cutoff=1.5,
                            pair=fsl.PAIR_SOFT, seed=8)
    b = fsl.Batch([other, cfg, other], [uniform_positions(30, (16,) * 3, 1), q,
                                       uniform_positions(60, (16,) * 3, 2)])
    o = oracle.Oracle(32, 32, 32, 32.0, 32.0, 32.0, q, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5,
                      kernel=3, pair=oracle.PAIR_SOFT, seed=7)
    b.step(3)
    o.step(3)
    b.sync()
    assert rel_inf(b.positions(1) - q, o.positions() - q) < 1e-4
    b.close()


def test_batch_large_planes_equal_alone(fsl):
    """Classes whose whole-plane transforms need more than 48 KB of shared
    memory (edges 72..128), two instances each, and a 5-7-11 edge."""
    inst = []
    for i, (m, k) in enumerate([(96, 3), (96, 3), (80, 4), (80, 4), (88, 3), (88, 3), (128, 4)]):
        cfg = fsl.make_config((m, m, m), (float(m),) * 3, eta=1.0 + 0.1 * i, kT=0.01, dt=0.01,
                              cutoff=1.5, kernel=k, pair=fsl.PAIR_SOFT, seed=500 + i)
        inst.append((cfg, uniform_positions(64 + 16 * i, (m, m, m), 70 + i)))
    b = fsl.Batch([c for c, _ in inst], [q for _, q in inst])
    b.step(2)
    b.sync()
    for i, (cfg, q) in enumerate(inst):
        qa, Fa, _ = run_alone(fsl, cfg, q, 2)
        np.testing.assert_array_equal(b.positions(i), qa)
    b.close()


def test_batch_mixed_pair_paths_equal_alone(fsl):
    """One size class holding a Verlet-list instance (soft), a cell-list one
    (LJ table, on a lattice), one without pair forces and a dense soft one
    that overflows its list into cell mode: every instance bitwise equal to
    the same instance alone, over steps with list rebuilds."""
    L = (20.0,) * 3
    g = np.arange(6) * 3.3 - 8.25
    lattice = np.stack(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1)
    rng = np.random.default_rng(5)
    dense = rng.uniform(-3.0, 3.0, (3, 600))
    cases = [
        (fsl.make_config((20,) * 3, L, kT=1.0, dt=0.02, cutoff=1.5, kernel=4, pair=fsl.PAIR_SOFT, seed=31),
         rng.uniform(-10, 10, (3, 300))),
        (fsl.make_config((20,) * 3, L, kT=0.01, dt=0.01, cutoff=1.5, kernel=4, pair=fsl.PAIR_TABLE_LJ, seed=32),
         lattice),
        (fsl.make_config((20,) * 3, L, kT=0.01, dt=0.01, cutoff=1.5, kernel=4, pair=fsl.PAIR_NONE, seed=33),
         rng.uniform(-10, 10, (3, 100))),
        (fsl.make_config((20,) * 3, L, kT=0.01, dt=0.01, cutoff=1.5, kernel=4, pair=fsl.PAIR_SOFT, seed=34),
         dense),
    ]
    b = fsl.Batch([c for c, _ in cases], [q for _, q in cases])
    assert b.info()["classes"] == 1
    b.step(12)
    b.sync()
    for i, (cfg, q) in enumerate(cases):
        qa, Fa, sa = run_alone(fsl, cfg, q, 12)
        np.testing.assert_array_equal(b.positions(i), qa)
        np.testing.assert_array_equal(b.forces(i), Fa)
        assert b.status(i)["error_bits"] == 0 and sa["error_bits"] == 0
    b.close()


def test_class_tuning_reports_picks(fsl):
    """Every size class reports the tuner's picks after its first step: the
    z-pass tile among the timed candidates, the faster transform schedule
    and, for a batch of small instances, the faster list build; a single
    instance reports the cooperative list build."""
    inst = mixed_set(fsl, n=12, np_max=2000)
    b = fsl.Batch([c for c, _ in inst], [q for _, q in inst])
    b.step(2)
    b.sync()
    tun = b.class_tuning()
    assert len(tun) == b.info()["classes"]
    assert sum(t["n"] for t in tun) == len(inst)
    for t in tun:
        assert t["tuned"] == 1
        assert t["fft_schedule"] in ("plane", "lines")
        assert t["z_tile_kx"] > 0 and t["z_tile_ky"] > 0 and t["z_threads"] > 0
        assert len(t["z_us"]) == t["z_candidates"] >= 1
        if t["z_candidates"] > 1:  # a single candidate is not timed
            assert all(u > 0 for u in t["z_us"])
        assert len(t["plane_us"]) == t["plane_candidates"] >= 1
        if t["plane_candidates"] > 1:
            assert all(u > 0 for u in t["plane_us"])
            best = min(range(t["plane_candidates"]), key=lambda i: t["plane_us"][i])
            assert t["plane_pb"] > 0 and t["plane_us"][best] == min(t["plane_us"])
        plane_us, lines_us = t["schedule_us"]
        if plane_us > 0 and lines_us > 0:  # both schedules exist for this edge
            assert t["fft_schedule"] == ("lines" if lines_us < plane_us else "plane")
        if t["n"] > 1:
            us_sep, us_blk = t["list_us"]
            assert us_sep > 0 and us_blk > 0
            assert t["list_build"] == ("block_per_instance" if us_blk <= us_sep else "separate")
    b.close()
    cfg, q = inst[0]
    g = fsl.StokesLimit(cfg, q)
    g.step(1)
    g.sync()
    t = g.tuning()
    assert t["tuned"] == 1 and t["list_build"] == "cooperative" and t["n"] == 1
    g.close()
