"""The serving loop through the fsl_server_* C ABI.

Requests submitted while others run are admitted at the next round and
share every launch with them; each result must still be bit-identical to the
same instance run alone through fsl_create/fsl_step.  Admission respects the
device-memory budget: with room for one slot, requests run one after another.
"""
import threading
import time

import numpy as np
import pytest

from helpers import uniform_positions

pytestmark = pytest.mark.gpu


def request_set(fsl, n, seed, edges=(16, 24, 32), np_max=300, steps=(1, 12)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        m = int(rng.choice(edges))
        npart = int(rng.integers(0, np_max)) if i % 5 else int(rng.integers(8, 40))
        kernel = int(rng.choice((3, 4)))
        cfg = fsl.make_config((m, m, m), (float(m),) * 3, eta=float(rng.uniform(0.5, 2.0)), kT=0.01,
                              dt=0.01, cutoff=1.5, kernel=kernel, pair=fsl.PAIR_SOFT,
                              seed=int(rng.integers(1, 1 << 40)))
        out.append((cfg, uniform_positions(npart, (m, m, m), 100 + i),
                    int(rng.integers(steps[0], steps[1] + 1))))
    return out


def run_alone(fsl, cfg, q, steps):
    g = fsl.StokesLimit(cfg, q)
    g.step(steps)
    g.sync()
    r = (g.positions(), g.forces())
    g.close()
    return r


def test_server_results_equal_alone(fsl):
    reqs = request_set(fsl, 12, seed=4)
    srv = fsl.Server(hbm_budget=4 << 30, max_round_steps=4)
    ids = [srv.submit(c, q, n) for c, q, n in reqs[:6]]
    time.sleep(0.05)  # the rest arrive while the first ones run
    ids += [srv.submit(c, q, n) for c, q, n in reqs[6:]]
    infos = [srv.wait(i, timeout=120) for i in ids]
    for info, (c, q, n) in zip(infos, reqs):
        assert info["state"] == fsl._lib.REQ_DONE, info
        assert info["steps_done"] == n and info["np"] == q.shape[1]
        assert info["submit_s"] <= info["start_s"] <= info["done_s"]
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["queued"] == 0
    assert st["steps"] == sum(n for _, _, n in reqs)
    for rid, (c, q, n) in zip(ids, reqs):
        qs, Fs = srv.result(rid)
        qa, Fa = run_alone(fsl, c, q, n)
        np.testing.assert_array_equal(qs, qa)
        np.testing.assert_array_equal(Fs, Fa)
    srv.close()


def test_server_concurrent_submitters(fsl):
    """submit/wait/result from several host threads at once."""
    reqs = request_set(fsl, 9, seed=9, edges=(16, 24), steps=(2, 6))
    srv = fsl.Server(hbm_budget=4 << 30)
    out = {}

    def client(k):
        c, q, n = reqs[k]
        rid = srv.submit(c, q, n)
        info = srv.wait(rid, timeout=120)
        out[k] = (info, srv.result(rid))

    th = [threading.Thread(target=client, args=(k,)) for k in range(len(reqs))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for k, (c, q, n) in enumerate(reqs):
        info, (qs, Fs) = out[k]
        assert info["state"] == fsl._lib.REQ_DONE
        qa, Fa = run_alone(fsl, c, q, n)
        np.testing.assert_array_equal(qs, qa)
    srv.close()


def test_server_budget_serializes_and_rejects(fsl):
    # room for one 16^3 slot (about 0.5 MB) but not two, nor a 32^3 one
    srv = fsl.Server(hbm_budget=700_000, max_round_steps=2)
    reqs = request_set(fsl, 3, seed=2, edges=(16,), np_max=60, steps=(3, 5))
    ids = [srv.submit(c, q, n) for c, q, n in reqs]
    big = fsl.make_config((32, 32, 32), (32.0,) * 3, kT=0.01, dt=0.01, cutoff=1.5,
                          pair=fsl.PAIR_SOFT)
    bid = srv.submit(big, uniform_positions(10, (32,) * 3, 1), 2)
    infos = [srv.wait(i, timeout=120) for i in ids]
    for a, b in zip(infos, infos[1:]):
        assert b["start_s"] >= a["done_s"]
    binfo = srv.wait(bid, timeout=120)
    assert binfo["state"] == fsl._lib.REQ_FAILED
    with pytest.raises(fsl._lib.FslError):
        srv.result(bid)
    for rid, (c, q, n) in zip(ids, reqs):
        qs, _ = srv.result(rid)
        np.testing.assert_array_equal(qs, run_alone(fsl, c, q, n)[0])
    assert srv.stats()["bytes_held"] <= 700_000
    srv.close()
