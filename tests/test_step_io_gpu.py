"""fsl_step_io: one step with its positions in from and out to host memory
gives the bits of fsl_set_positions + fsl_step(1) + fsl_get_positions.

With page-locked buffers both copies are nodes of the step's graph and the
copy in runs beside the noise; with pageable buffers the three calls run.
Between steps the host moves the particles (some by more than half the
Verlet skin, so the moved check inside the graph requests list rebuilds),
as a caller coupling the step to host-side work would.
"""
import numpy as np
import pytest

from helpers import uniform_positions

pytestmark = pytest.mark.gpu


def _config(fsl):
    return fsl.make_config((48, 48, 48), (48.0,) * 3, kT=0.01, dt=0.01, cutoff=1.5, kernel=4,
                           pair=fsl.PAIR_SOFT, seed=41)


def _host_moves(q, rng, k):
    """Small moves every step, a few large ones every third step."""
    q += rng.normal(0.0, 0.01, q.shape)
    if k % 3 == 2:
        idx = rng.choice(q.shape[1], 20, replace=False)
        q[:, idx] += rng.normal(0.0, 0.5, (3, 20))


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_step_io_equals_set_step_get(fsl, pinned):
    import torch
    cfg = _config(fsl)
    q0 = uniform_positions(6000, (48, 48, 48), 7)
    a = fsl.StokesLimit(cfg, q0)
    b = fsl.StokesLimit(cfg, q0)
    if pinned:
        buf = torch.empty((3, q0.shape[1]), dtype=torch.float64).pin_memory()
        qa = buf.numpy()
    else:
        qa = np.empty_like(q0)
    qa[...] = q0
    qb = q0.copy()
    rng_a, rng_b = np.random.default_rng(3), np.random.default_rng(3)
    for k in range(9):
        a.step_io(qa, qa)
        b.set_positions(qb)
        b.step(1)
        qb = b.positions()
        np.testing.assert_array_equal(qa, qb)
        _host_moves(qa, rng_a, k)
        _host_moves(qb, rng_b, k)
    np.testing.assert_array_equal(a.forces(), b.forces())
    np.testing.assert_array_equal(a.velocity(), b.velocity())
    sa, sb = a.status(), b.status()
    assert sa["step"] == sb["step"] == 9 and sa["error_bits"] == sb["error_bits"] == 0
    if pinned:
        assert sa["graph"]
    a.close()
    b.close()


def test_step_io_then_plain_steps(fsl):
    """Alternating the input/output step with plain steps (each change of
    step kind captures its graph again) keeps the bits of the plain calls."""
    import torch
    cfg = _config(fsl)
    q0 = uniform_positions(3000, (48, 48, 48), 8)
    a = fsl.StokesLimit(cfg, q0)
    b = fsl.StokesLimit(cfg, q0)
    buf = torch.empty((3, q0.shape[1]), dtype=torch.float64).pin_memory()
    qa = buf.numpy()
    qa[...] = q0
    rng = np.random.default_rng(5)
    for k in range(4):
        q_in = qa.copy()
        a.step_io(qa, qa)
        a.step(2)
        b.set_positions(q_in)
        b.step(3)
        np.testing.assert_array_equal(a.positions(), b.positions())
        qa[...] = a.positions() + rng.normal(0.0, 0.01, qa.shape)
    a.close()
    b.close()


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_batch_step_io_equals_set_step_get(fsl, pinned):
    """The batched form: every instance of a batch over three size classes
    (one instance empty) bit for bit as the packed set, step and get."""
    import torch
    rng = np.random.default_rng(9)
    cfgs, qs = [], []
    for i in range(9):
        m = (16, 24, 32)[i % 3]
        n = 0 if i == 4 else 200 + 150 * i
        cfgs.append(fsl.make_config((m, m, m), (float(m),) * 3, kT=0.01, dt=0.01, cutoff=1.5,
                                    kernel=3 + i % 2, pair=fsl.PAIR_SOFT, seed=60 + i))
        qs.append(uniform_positions(n, (m, m, m), 20 + i))
    a = fsl.Batch(cfgs, qs)
    b = fsl.Batch(cfgs, qs)
    n = int(a.offsets[-1])
    if pinned:
        buf = torch.empty(n, dtype=torch.float64).pin_memory()
        qa = buf.numpy()
    else:
        qa = np.empty(n)
    a.positions_packed(qa)
    qb = qa.copy()
    for k in range(6):
        a.step_io(qa, qa)
        b.set_positions_packed(qb)
        b.step(1)
        b.positions_packed(qb)
        np.testing.assert_array_equal(qa, qb)
        moves = rng.normal(0.0, 0.01, n)
        qa += moves
        qb += moves
    for i in range(len(cfgs)):
        np.testing.assert_array_equal(a.forces(i), b.forces(i))
        assert a.status(i)["error_bits"] == b.status(i)["error_bits"] == 0
    a.close()
    b.close()
