"""Shared helpers of the test suite (seeded synthetic inputs, error norms)."""
import numpy as np


def uniform_positions(n, box, seed):
    rng = np.random.default_rng(seed)
    L = np.asarray(box, dtype=float).reshape(3, 1)
    return rng.uniform(-0.5, 0.5, (3, n)) * L


def chains(nchains, beads, box, seed, r0=1.0):
    """Bead-spring chains: seeded uniform starts, each bond a seeded random
    unit vector of length r0.  Returns positions (3, np) and bond lists."""
    rng = np.random.default_rng(seed)
    L = np.asarray(box, dtype=float)
    starts = rng.uniform(-0.5, 0.5, (nchains, 3)) * L
    d = rng.standard_normal((nchains, beads - 1, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    pos = np.concatenate([starts[:, None, :], starts[:, None, :] + np.cumsum(d * r0, axis=1)], axis=1)
    q = pos.reshape(-1, 3).T.copy()
    idx = np.arange(nchains * beads).reshape(nchains, beads)
    bi = idx[:, :-1].ravel().astype(np.int32)
    bj = idx[:, 1:].ravel().astype(np.int32)
    return q, bi, bj


def rel_inf(a, b):
    """max |a - b| / max |b|"""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
