"""The W build fused into the first pass of the register plane transform
(the default where that path exists) against the separate W build
(FLUAMSL_FUSED_W=0): the same W arithmetic, so the runs agree to FP32
rounding of the stress-divergence sums."""
import os

import numpy as np
import pytest

from helpers import chains, uniform_positions

pytestmark = pytest.mark.gpu


def _run(fsl, m, L, n, kernel, fused, precision=0, steps=5, scheme=0):
    q = uniform_positions(n, (L,) * 3, 13)
    cfg = fsl.make_config((m,) * 3, (L,) * 3, eta=1.0, kT=0.01, dt=0.01, cutoff=1.5, kernel=kernel,
                          pair=fsl.PAIR_SOFT, soft_epsilon=1.0, seed=23, precision=precision, scheme=scheme)
    old = os.environ.get("FLUAMSL_FUSED_W")
    os.environ["FLUAMSL_FUSED_W"] = "1" if fused else "0"
    try:
        with fsl.StokesLimit(cfg, q) as s:
            s.step(steps)
            assert s.status()["error_bits"] == 0
            return s.positions(), s.velocity64(), q
    finally:
        if old is None:
            del os.environ["FLUAMSL_FUSED_W"]
        else:
            os.environ["FLUAMSL_FUSED_W"] = old


# register plane edges: 16 and 24 stage the plane in shared memory (T = 1),
# the others hold lines in registers
@pytest.mark.parametrize("m,kernel", [(16, 3), (24, 4), (32, 4), (48, 3), (64, 4), (96, 3), (128, 4)])
def test_fused_w_matches_separate(fsl, m, kernel):
    n = min(400, m ** 3 // 40)
    q0, v0, qi = _run(fsl, m, float(m), n, kernel, False)
    q1, v1, _ = _run(fsl, m, float(m), n, kernel, True)
    dq = np.abs(q0 - qi).max()
    assert np.abs(q1 - q0).max() <= 1e-5 * dq
    assert np.abs(v1 - v0).max() <= 1e-5 * np.abs(v0).max()


def test_fused_w_first_order_and_float_atomic(fsl):
    for kw in (dict(scheme=1), dict(precision=1)):
        q0, v0, qi = _run(fsl, 32, 32.0, 300, 4, False, **kw)
        q1, v1, _ = _run(fsl, 32, 32.0, 300, 4, True, **kw)
        dq = np.abs(q0 - qi).max()
        assert np.abs(q1 - q0).max() <= 1e-5 * dq
        assert np.abs(v1 - v0).max() <= 1e-5 * np.abs(v0).max()
