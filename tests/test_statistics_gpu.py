"""Statistical checks of the GPU step beside the oracle parity.

1. Single-particle mobility J L^-1 P S of the 3- and 4-point kernels against
   the periodic Hasimoto expansion mu(L) = (1 - 2.837297 a/L + 4.19 (a/L)^3
   - 27.4 (a/L)^6) / (6 pi eta a): one hydrodynamic radius a fits two box
   sizes, and it is the kernel's known one (3-point 0.9108 dx, 4-point
   1.2527 dx; the FP64 oracle gives the same to 1e-4).
2. Equilibrium velocity variance: free particles in thermal equilibrium move
   per step with <dq_a^2> = 2 kT mu dt per component (<u_a^2> = 2 kT mu / dt
   for the velocity u = dq / dt), mu the self mobility of 1.
"""
import numpy as np
import pytest

from helpers import uniform_positions

pytestmark = pytest.mark.gpu

A_H = {3: 0.9108, 4: 1.2527}


def hasimoto(a, L, eta=1.0):
    x = a / L
    return (1 - 2.837297 * x + 4.19 * x ** 3 - 27.4 * x ** 6) / (6 * np.pi * eta * a)


def fit_radius(mu, L):
    from scipy.optimize import brentq
    return brentq(lambda a: hasimoto(a, L) - mu, 0.3, 3.0)


def mobility(fsl, kernel, L, offsets):
    cfg = fsl.make_config((L, L, L), (float(L),) * 3, eta=1.0, kT=0.0, dt=0.01, cutoff=1.5,
                          kernel=kernel, pair=fsl.PAIR_NONE, seed=1)
    out = []
    with fsl.StokesLimit(cfg, np.array([[0.1], [0.2], [0.3]])) as s:
        for off in offsets:
            s.set_positions(np.asarray(off, dtype=float).reshape(3, 1))
            for d in range(3):
                F = np.zeros((3, 1))
                F[d, 0] = 1.0
                u = s.interpolate(s.solve(s.spread(F)))
                out.append(u[d, 0])
    return float(np.mean(out))


@pytest.mark.parametrize("kernel", [3, 4])
def test_mobility_hasimoto(fsl, kernel):
    rng = np.random.default_rng(4)
    offsets = rng.uniform(-0.5, 0.5, size=(8, 3))
    radii = []
    for L in (32, 64):
        mu = mobility(fsl, kernel, L, offsets)
        radii.append(fit_radius(mu, L))
    assert abs(radii[0] - radii[1]) < 2e-3 * radii[0]
    assert abs(np.mean(radii) / A_H[kernel] - 1) < 5e-3


@pytest.mark.parametrize("kernel", [3, 4])
def test_equilibrium_velocity_variance(fsl, kernel):
    L, kT, dt, steps = 64, 1.0, 0.01, 20
    g = np.arange(8) * 8.0 - 28.0
    q = np.stack(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1)
    q = q + uniform_positions(q.shape[1], (4.0,) * 3, 6)  # off the grid nodes
    cfg = fsl.make_config((L, L, L), (float(L),) * 3, eta=1.0, kT=kT, dt=dt, cutoff=1.5,
                          kernel=kernel, pair=fsl.PAIR_NONE, seed=12, observables=1)
    d2 = []
    with fsl.StokesLimit(cfg, q) as s:
        prev = s.positions()
        for _ in range(steps):
            s.step(1)
            cur = s.positions()
            d2.append((cur - prev) ** 2)
            prev = cur
        obs = s.observables()
    d2 = np.concatenate(d2, axis=1)  # 3 x (512 particles * 20 steps)
    mu = hasimoto(A_H[kernel], L)
    u2 = d2.mean() / dt ** 2
    # 30,720 samples: the estimator's relative spread is about 1%
    assert abs(u2 / (2 * kT * mu / dt) - 1) < 0.05
    # per component too, and the device MSD accumulator follows the diffusion
    for a in range(3):
        assert abs(d2[a].mean() / (2 * kT * mu * dt) - 1) < 0.08
    assert obs["steps"] == steps
    assert abs(obs["msd"] / (6 * kT * mu * dt * steps) - 1) < 0.25
