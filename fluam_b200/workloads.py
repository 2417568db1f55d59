"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No dataset is involved: particle positions are seeded uniform (or seeded
bead-spring chains) and the noise is drawn on the device from the seed.

  plain_32   32^3 cells, dx = 1, eta 1, kT 0.01, dt 0.01, 3-pt kernel,
             256 uniform particles, soft repulsion eps 1, rc 1.5
  plain_128  128^3 cells, dx = 1, eta 1, kT 0.01, dt 0.005, 4-pt kernel,
             65,536 particles = 4,096 chains x 16 beads, harmonic bonds k 10,
             r0 1 (chain starts seeded uniform, each bond a seeded random unit
             vector), soft repulsion eps 1, rc 1.5
  mixed_1024 1,024 independent periodic cubic replicas, dx = 1: edge uniform
             over {16, 24, 32, 48, 64}, np = round(exp(U[ln 8, ln 2048])) seeded
             uniform positions, eta ~ U[0.5, 2], kT 0.01, dt 0.01, 3-pt kernel,
             soft repulsion eps 1, rc 1.5, one seed per replica
"""
import numpy as np

from . import PAIR_SOFT, make_config

WORKLOADS = {
    "plain_32": dict(cells=32, box=32.0, eta=1.0, kT=0.01, dt=0.01, kernel=3, n=256,
                     chains=0, beads=0, k=0.0, r0=0.0, eps=1.0, rc=1.5),
    "plain_128": dict(cells=128, box=128.0, eta=1.0, kT=0.01, dt=0.005, kernel=4, n=65536,
                      chains=4096, beads=16, k=10.0, r0=1.0, eps=1.0, rc=1.5),
}


def uniform(n, box, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-0.5, 0.5, (3, n)) * float(box)


def chains(nchains, beads, box, seed, r0=1.0):
    """Bead-spring chains; returns positions (3, np) and the bond index lists."""
    rng = np.random.default_rng(seed)
    starts = rng.uniform(-0.5, 0.5, (nchains, 3)) * float(box)
    d = rng.standard_normal((nchains, beads - 1, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    pos = np.concatenate([starts[:, None, :], starts[:, None, :] + np.cumsum(d * r0, axis=1)],
                         axis=1)
    q = pos.reshape(-1, 3).T.copy()
    idx = np.arange(nchains * beads).reshape(nchains, beads)
    return q, idx[:, :-1].ravel().astype(np.int32), idx[:, 1:].ravel().astype(np.int32)


def build(name, seed=1):
    """(config, positions, bonds or None) of a named workload."""
    w = WORKLOADS[name]
    m, L = w["cells"], w["box"]
    cfg = make_config((m, m, m), (L, L, L), eta=w["eta"], kT=w["kT"], dt=w["dt"], cutoff=w["rc"],
                      kernel=w["kernel"], pair=PAIR_SOFT, soft_epsilon=w["eps"], seed=seed)
    if w["chains"]:
        q, bi, bj = chains(w["chains"], w["beads"], L, seed, w["r0"])
        nb = len(bi)
        bonds = (bi, bj, np.full(nb, w["k"]), np.full(nb, w["r0"]))
    else:
        q, bonds = uniform(w["n"], L, seed), None
    return cfg, q, bonds


MIXED_EDGES = (16, 24, 32, 48, 64)


def mixed(n=1024, seed=7, edges=MIXED_EDGES, np_range=(8, 2048)):
    """Replica set of the batched workload: a list of (config, positions)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        m = int(rng.choice(edges))
        npart = int(round(np.exp(rng.uniform(np.log(np_range[0]), np.log(np_range[1])))))
        eta = float(rng.uniform(0.5, 2.0))
        cfg = make_config((m, m, m), (float(m),) * 3, eta=eta, kT=0.01, dt=0.01, cutoff=1.5,
                          kernel=3, pair=PAIR_SOFT, soft_epsilon=1.0, seed=seed * 100003 + i)
        out.append((cfg, uniform(npart, m, seed * 7919 + i)))
    return out
