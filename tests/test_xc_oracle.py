"""The local functionals' CPU restatement (oracle/xc.py) against nAPMO's own
LDA fixtures (napmo/functional/test, produced through LibXC; subsampled into
tests/golden/xc_lda.npz by tests/golden/make_xc_golden.py)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'xc_lda.npz')


def test_lda_restatement_matches_napmo_fixtures():
    import xc
    g = np.load(GOLDEN)
    zx, vx = xc.lda_x(g['rho'])
    zc, vc = xc.lda_c_vwn(g['rho'])
    assert np.abs(zx - g['x_zk']).max() <= 1e-15 * np.abs(g['x_zk']).max()
    assert np.abs(vx - g['x_vrho']).max() <= 1e-15 * np.abs(g['x_vrho']).max()
    assert np.abs(zc - g['c_zk']).max() <= 1e-15
    assert np.abs(vc - g['c_vrho']).max() <= 1e-15
    # the cut of the smallest densities: zero below, nonzero from 1.2e-22 up
    assert np.all(g['x_zk'][g['rho'] < 1e-24] == 0.0)
    assert np.all(zx[g['rho'] < 1e-24] == 0.0)


def test_lda_potentials_are_derivatives_of_the_energy_density():
    import xc
    rho = np.geomspace(1e-8, 50.0, 200)
    h = 1e-6 * rho
    for f in (xc.lda_x, xc.lda_c_vwn):
        zk, v = f(rho)
        ep = f(rho + h)[0] * (rho + h)
        em = f(rho - h)[0] * (rho - h)
        assert np.abs((ep - em) / (2 * h) - v).max() <= 1e-7 * np.abs(v).max()


def test_epc17_2_branches():
    import xc
    rng = np.random.default_rng(3)
    e, n = rng.random(50) + 0.1, rng.random(50) + 0.1
    ene, pa, pb = xc.epc17_2(e, n)
    den = 2.35 - 2.4 * np.sqrt(e * n) + 6.6 * e * n
    assert np.allclose(ene, -n / den, rtol=1e-15, atol=0)
    # pa is d(e * ene)/d(rho_E) in the regular branch
    h = 1e-7
    f = lambda x: x * xc.epc17_2(x, n)[0]
    assert np.allclose((f(e + h) - f(e - h)) / (2 * h), pa, rtol=1e-6)
    e2 = e.copy()
    e2[0] = 0.0                       # a zero density switches every point
    _, pa2, _ = xc.epc17_2(e2, n)
    den2 = 2.35 - 2.4 * np.sqrt(e2 * n) + 6.6 * e2 * n
    assert np.allclose(pa2, (2.4 * np.sqrt(e2) * n ** 1.5 - 2 * 2.35 * n) / den2 ** 2 / 2)


def test_polarised_lda_at_zero_spin_matches_napmo_fixtures():
    """With rho_a = rho_b = rho / 2 the spin-polarised restatement gives
    nAPMO's own (unpolarised, LibXC) fixtures: exchange to rounding,
    correlation exactly (f(0) = f'(0) = 0 leaves the paramagnetic fit)."""
    import xc
    g = np.load(GOLDEN)
    rho = g['rho']
    zx, va, vb = xc.lda_x_polarized(rho / 2, rho / 2)
    zc, ca, cb = xc.lda_c_vwn_polarized(rho / 2, rho / 2)
    assert np.abs(zx - g['x_zk']).max() <= 1e-15 * np.abs(g['x_zk']).max()
    assert np.abs(va - g['x_vrho']).max() <= 1e-15 * np.abs(g['x_vrho']).max()
    assert np.array_equal(va, vb)
    assert np.abs(zc - g['c_zk']).max() <= 1e-15
    assert np.abs(ca - g['c_vrho']).max() <= 1e-15
    assert np.array_equal(ca, cb)


def test_polarised_lda_potentials_and_limits():
    """Spin potentials are the derivatives of the energy density
    rho e(rho_a, rho_b); fully polarised exchange is 2^(1/3) times the
    unpolarised one at the same total density; the VWN fits give the known
    values at r_s = 1 (paramagnetic -0.0600, ferromagnetic -0.0315 Eh)."""
    import xc
    rng = np.random.default_rng(5)
    ra, rb = rng.uniform(1e-4, 5.0, 100), rng.uniform(1e-4, 5.0, 100)
    for f in (xc.lda_x_polarized, xc.lda_c_vwn_polarized):
        zk, va, vb = f(ra, rb)
        E = lambda a, b: f(a, b)[0] * (a + b)
        ha, hb = 1e-6 * ra, 1e-6 * rb
        fa = (E(ra + ha, rb) - E(ra - ha, rb)) / (2 * ha)
        fb = (E(ra, rb + hb) - E(ra, rb - hb)) / (2 * hb)
        assert np.abs(fa - va).max() <= 1e-7 * np.abs(va).max()
        assert np.abs(fb - vb).max() <= 1e-7 * np.abs(vb).max()
    rho = np.geomspace(1e-6, 50.0, 50)
    assert np.allclose(xc.lda_x_polarized(rho, 0 * rho)[0] / xc.lda_x(rho)[0], 2 ** (1 / 3),
                       rtol=1e-15, atol=0)
    x = 1.0
    eP = xc._vwn_fit(x, xc.VWN_A, xc.VWN_B, xc.VWN_C, xc.VWN_X0)[0]
    eF = xc._vwn_fit(x, *xc.VWN_F)[0]
    assert abs(eP + 0.0600) < 1e-4 and abs(eF + 0.0315) < 1e-4
    # below the cut, and negative spin densities count as zero
    z = xc.lda_c_vwn_polarized(np.array([1e-25, 1.0]), np.array([1e-26, -1e-3]))
    assert z[0][0] == 0.0 and np.isfinite(z[0][1])
    assert np.allclose(z[0][1], xc.lda_c_vwn_polarized(1.0, 0.0)[0])
