"""Known-answer tests of the FP64 CPU oracle (no GPU).

The reference ships no tests or golden vectors for this path; these identities
pin the oracle's pieces from first principles, and tests/test_oracle_vs_ref.py
pins the whole step against the reference's own sources compiled for the host.
"""
import numpy as np
import pytest

from helpers import chains, rel_inf, uniform_positions


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 10, 12), (7, 11, 13), (24, 40, 16), (5, 9, 22)])
def test_fft_matches_numpy(oracle, shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert np.abs(oracle.fft3d(a, -1) - np.fft.fftn(a)).max() < 1e-11 * a.size ** 0.5
    assert np.abs(oracle.fft3d(a, +1) - np.fft.ifftn(a) * a.size).max() < 1e-11 * a.size ** 0.5


def test_noise_moments_and_determinism(oracle):
    n = oracle.noise(123, 4, 0, 400000)
    assert abs(n.mean()) < 0.01 and abs(n.var() - 1) < 0.01
    assert abs(((n ** 4).mean()) - 3.0) < 0.05
    np.testing.assert_array_equal(n[1000:1010], oracle.noise(123, 4, 1000, 10))
    assert not np.allclose(n[:100], oracle.noise(123, 5, 0, 100))
    assert not np.allclose(n[:100], oracle.noise(124, 4, 0, 100))
    # consecutive indices within one Philox block are not correlated
    assert abs(np.corrcoef(n[0::4], n[1::4])[0, 1]) < 0.02


@pytest.mark.parametrize("x0", [0.0, 0.13, 0.37, 0.5, -0.21, 0.49999])
def test_peskin3_moments(oracle, x0):
    j = np.arange(-3, 4)
    w = np.array([oracle.delta3(x0 - k) for k in j])
    assert abs(w.sum() - 1) < 1e-6  # sqrtf in the reference's kernel
    assert abs((w * (x0 - j)).sum()) < 1e-6
    assert abs((w ** 2).sum() - 0.5) < 1e-6


@pytest.mark.parametrize("x0", [0.0, 0.13, 0.37, 0.5, 0.77, 0.999])
def test_peskin4_moments(oracle, x0):
    j = np.arange(-3, 5)
    w = np.array([oracle.delta4(x0 - k) for k in j])
    assert abs(w.sum() - 1) < 1e-13
    assert abs((w * (x0 - j)).sum()) < 1e-13
    assert abs((w ** 2).sum() - 3.0 / 8.0) < 1e-13
    assert abs(w[j % 2 == 0].sum() - 0.5) < 1e-13


def _oracle(oracle, m=(16, 12, 8), L=(16.0, 12.0, 8.0), q=None, **kw):
    if q is None:
        q = np.zeros((3, 1))
    return oracle.Oracle(m[0], m[1], m[2], L[0], L[1], L[2], q, **kw)


def test_single_mode_shear_wave(oracle):
    """A divergence-free shear wave W_x(y) is returned as W/(eta g_y^2)."""
    mx, my, mz = 16, 12, 8
    eta = 1.7
    o = _oracle(oracle, eta=eta)
    ky = 3
    y = np.arange(my)
    W = np.zeros((3, mz, my, mx))
    W[0] = np.cos(2 * np.pi * ky * y / my)[None, :, None]
    v = o.solve(W)
    gy = 2.0 * np.sin(np.pi * ky / my)  # dy = 1
    np.testing.assert_allclose(v[0], W[0] / (eta * gy ** 2), atol=1e-12)
    assert np.abs(v[1:]).max() < 1e-12


def test_single_mode_compressional_is_projected_out(oracle):
    mx, my, mz = 16, 12, 8
    o = _oracle(oracle)
    kx = 2
    x = np.arange(mx) + 0.5  # x-faces
    W = np.zeros((3, mz, my, mx))
    W[0] = np.cos(2 * np.pi * kx * x / mx)[None, None, :]
    v = o.solve(W)
    assert np.abs(v).max() < 1e-12


def test_solve_divergence_free_and_zero_mean(oracle):
    o = _oracle(oracle)
    W = np.random.default_rng(3).standard_normal((3, 8, 12, 16))
    v = o.solve(W)
    div = (v[0] - np.roll(v[0], 1, axis=2)) + (v[1] - np.roll(v[1], 1, axis=1)) + \
        (v[2] - np.roll(v[2], 1, axis=0))
    assert np.abs(div).max() < 1e-12
    assert np.abs(v.mean(axis=(1, 2, 3))).max() < 1e-13


@pytest.mark.parametrize("kernel", [3, 4])
def test_spread_interp_adjoint(oracle, kernel):
    """<J v, F> = dV <v, S F>: interpolation is the adjoint of spreading."""
    L = (16.0, 12.0, 8.0)
    m = (32, 24, 16)  # dx = 0.5
    q = uniform_positions(40, L, 7) * 1.7  # unwrapped positions too
    o = _oracle(oracle, m=m, L=L, q=q, kernel=kernel)
    rng = np.random.default_rng(8)
    F = rng.standard_normal((3, 40))
    v = rng.standard_normal((3, m[2], m[1], m[0]))
    dV = 0.5 ** 3
    lhs = (o.interp(q, v) * F).sum()
    rhs = dV * (v * o.spread(q, F)).sum()
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


@pytest.mark.parametrize("kernel", [3, 4])
def test_spread_conserves_force(oracle, kernel):
    L = (12.0, 12.0, 12.0)
    q = uniform_positions(30, L, 2)
    o = _oracle(oracle, m=(12, 12, 12), L=L, q=q, kernel=kernel)
    F = np.random.default_rng(4).standard_normal((3, 30))
    f = o.spread(q, F)
    np.testing.assert_allclose(f.sum(axis=(1, 2, 3)), F.sum(axis=1), rtol=1e-6, atol=1e-9)


def test_cell_list_is_counting_sort(oracle):
    L = (20.0, 20.0, 20.0)
    q = uniform_positions(500, L, 11)
    q[:, :10] += 40.0  # unwrapped coordinates
    o = _oracle(oracle, m=(20, 20, 20), L=L, q=q, cutoff=1.5)
    (mnx, mny, mnz), M = o.neighbor_grid()
    assert (mnx, mny, mnz) == (13, 13, 13) and M == 13 ** 3
    cell_of, start, srt = o.cell_list(q)
    # brute-force cell index of the wrapped coordinate
    w = q - np.trunc(q / 20.0 + 0.5 * np.sign(q)) * 20.0
    j = (np.trunc(w * (13 / 20.0) + 6.5).astype(int)) % 13
    np.testing.assert_array_equal(cell_of, j[0] + 13 * j[1] + 169 * j[2])
    assert start[0] == 0 and start[-1] == 500
    np.testing.assert_array_equal(np.diff(start), np.bincount(cell_of, minlength=M))
    for c in range(M):
        members = srt[start[c]:start[c + 1]]
        assert np.all(np.diff(members) > 0) and np.all(cell_of[members] == c)


def _brute_soft(q, L, rc, eps):
    d = q[:, :, None] - q[:, None, :]
    d -= np.round(d / L[:, None, None]) * L[:, None, None]
    r = np.sqrt((d ** 2).sum(axis=0))
    np.fill_diagonal(r, np.inf)
    f = np.where(r < rc, (2 * eps / rc) * (1 - r / rc) / r, 0.0)
    return (f[None] * d).sum(axis=2)


def test_soft_repulsion_matches_brute_force(oracle):
    L = np.array([10.0, 10.0, 10.0])
    q = uniform_positions(300, L, 5)
    o = _oracle(oracle, m=(10, 10, 10), L=tuple(L), q=q, cutoff=1.5, pair=oracle.PAIR_SOFT,
                soft_epsilon=1.3)
    F = o.compute_forces(q)
    np.testing.assert_allclose(F, _brute_soft(q, L, 1.5, 1.3), rtol=1e-12, atol=1e-12)


def test_lj_table_emulation(oracle):
    L = (32.0, 32.0, 32.0)
    rc = 2 ** (1 / 6) * 2.0
    o = _oracle(oracle, m=(32, 32, 32), L=L, cutoff=rc, pair=oracle.PAIR_TABLE_LJ, kT=0.5)
    tab = o.ljtable()
    assert tab[0] == 0 and tab[-1] == 0
    # the reference accumulates r^2 in single precision (src/initForcesNonBonded.cu:39-45)
    dr = np.float32(np.float32(rc * rc) / np.float32(4096))
    r2 = np.empty(4096, np.float32)
    acc = np.float32(0.5) * dr
    for i in range(4096):
        r2[i] = acc
        acc = np.float32(acc + dr)
    rr32 = np.sqrt(r2)  # single-precision sqrt, as sqrt(float) in the reference
    rr = rr32.astype(np.float64)
    fr = (48 * 0.5 * ((2 / rr) ** 12 - 0.5 * (2 / rr) ** 6) / rr).astype(np.float32)
    lj = fr / rr32
    np.testing.assert_allclose(tab[1:-1], lj[1:-1], rtol=1e-7)
    # and the table is the LJ force / r up to single-precision rounding
    ljx = 48 * 0.5 * ((2 / rr) ** 12 - 0.5 * (2 / rr) ** 6) / rr ** 2
    assert rel_inf(tab[1:-1], ljx[1:-1]) < 1e-6
    # at a texel centre the filter returns the entry itself
    for i in (5, 100, 2047, 4000):
        x = np.float32((i + 0.5) / 4096)
        assert oracle.tex_linear(tab, x) == tab[i]
    # half way between texels: the mean of the two
    x = np.float32((100 + 1.0) / 4096)
    assert abs(oracle.tex_linear(tab, x) - 0.5 * (tab[100] + tab[101])) <= 1e-6 * abs(tab[100])
    # clamped at both ends
    assert oracle.tex_linear(tab, np.float32(0.0)) == tab[0]
    assert oracle.tex_linear(tab, np.float32(2.0)) == tab[-1]


def test_bonds_and_tethers(oracle):
    L = (30.0, 30.0, 30.0)
    q, bi, bj = chains(3, 5, L, 9)
    n = q.shape[1]
    o = _oracle(oracle, m=(30, 30, 30), L=L, q=q, cutoff=1.5, pair=oracle.PAIR_NONE)
    k = np.full(len(bi), 10.0)
    r0 = np.where(np.arange(len(bi)) % 2 == 0, 1.0, 0.0)
    fxyz = np.array([[0.5, -1.0, 2.0]])
    o.set_bonds(bi, bj, k, r0, fi=[2], fk=[3.0], fr0=[0.0], fxyz=fxyz)
    F = o.compute_forces(q)
    ref = np.zeros((3, n))
    for a, b, kk, rr in zip(bi, bj, k, r0):
        d = q[:, a] - q[:, b]
        r = np.linalg.norm(d)
        f = -kk * (1 - rr / r) * d if rr != 0 else -kk * d
        ref[:, a] += f
        ref[:, b] -= f
    ref[:, 2] += -3.0 * (q[:, 2] - fxyz[0])
    np.testing.assert_allclose(F, ref, rtol=1e-12, atol=1e-12)
    with pytest.raises(ValueError):
        o.set_bonds([0], [n], [1.0], [1.0])


def test_step_statistics_free_particles(oracle):
    """Mean square displacement of free particles follows 2 kT mu dt with the
    periodic Hasimoto mobility of the 3-point kernel (a_h ~ 0.91 dx)."""
    L = (32.0, 32.0, 32.0)
    q = uniform_positions(64, L, 21) * 0.0
    q = np.stack(np.meshgrid(*[np.arange(4) * 8.0 - 12.0] * 3, indexing="ij")).reshape(3, -1)
    q = q + 0.3
    o = _oracle(oracle, m=(32, 32, 32), L=L, q=q, kT=0.01, dt=0.01, pair=oracle.PAIR_NONE,
                cutoff=1.5, seed=5)
    disp = []
    for _ in range(40):
        q0 = o.positions()
        o.step(1)
        disp.append(o.positions() - q0)
    d2 = np.mean(np.concatenate(disp, axis=1) ** 2)
    ah = 0.91
    mu = 1 / (6 * np.pi * ah) * (1 - 2.837297 * ah / 32 + 4.19 * (ah / 32) ** 3)
    expect = 2 * 0.01 * mu * 0.01
    # 64 particles x 40 steps x 3 components; hydrodynamic correlations widen it
    assert abs(d2 / expect - 1) < 0.12


def test_fp32_build_tracks_fp64(oracle):
    """The FP32 build of the restatement (the CPU timing baseline in single
    precision, `double` replaced by `float` as the reference's own FP32 route
    does) follows the FP64 build: 3 midpoint steps of 256 particles at 32^3."""
    q = uniform_positions(256, (32.0,) * 3, 5)
    a = oracle.Oracle(32, 32, 32, 32.0, 32.0, 32.0, q, kernel=3, seed=3)
    b = oracle.Oracle(32, 32, 32, 32.0, 32.0, 32.0, q, kernel=3, seed=3, real="f32")
    a.step(3)
    b.step(3)
    assert b.positions().dtype == np.float32
    assert rel_inf(b.positions() - q, a.positions() - q) < 1e-3
