"""The int8-slice scheme of the mixed-precision path, on the CPU.

oracle/ozaki.py restates the scheme the tensor-core kernels implement; these
tests pin its accuracy against exact FP64 contractions on small grids, so the
GPU tests can compare the kernels with it exactly.
"""
import numpy as np
import pytest

from helpers import H2O, oracle_system, random_density


@pytest.fixture(scope='module')
def h2o_case(oracle, basis_library, elements):
    g, fb = oracle_system(oracle, basis_library, elements, H2O, nrad=30, nang=50)
    phi = oracle.basis_compute(fb, g.points).T.copy()
    D = random_density(phi.shape[0], 5)
    rho = oracle.density(phi, D)
    v = oracle.compute_coulomb(g, rho, 5)
    return g, phi, D, rho, v


def test_digits_roundtrip():
    import ozaki
    rng = np.random.default_rng(3)
    x = rng.normal(size=(7, 1000)) * np.exp(rng.uniform(-30, 5, size=(7, 1)))
    e = ozaki.group_exponent(np.abs(x).max(axis=1))
    d = ozaki.digits(x, e[:, None])
    assert np.abs(d[0]).max() <= 64
    for k in range(1, 4):
        assert d[k].min() >= -128 and d[k].max() <= 127
    Y = ((d[0] * 256 + d[1]) * 256 + d[2]) * 256 + d[3]
    back = np.ldexp(Y.astype(np.float64), (e[:, None] - 30))
    # one rounding: half an ulp of 2^(e - 30)
    assert np.all(np.abs(back - x) <= np.ldexp(0.5, e[:, None] - 30))


def test_balance_is_power_of_two():
    import ozaki
    t = np.array([1e-12, 3.7e-5, 1.0, 2.0, 17.5, 0.0, -1.0, -8.05e-6])
    sc, isc = ozaki.balance(t, np.ones_like(t))
    assert np.all(sc * isc == 1.0)
    assert np.all(np.frexp(sc)[0] == 0.5)
    nz = t != 0
    # c = floor(log2 |t| / 2): |t| / sc^2 in [1, 4), negative weights included
    r = np.abs(t[nz]) / sc[nz] ** 2
    assert np.all((r >= 1.0) & (r < 4.0))
    assert sc[t == 0][0] == 1.0


def test_scheme_quadrature_accuracy(h2o_case):
    import ozaki
    g, phi, D, rho, v = h2o_case
    wv = g.becke * g.weights * v
    F64 = (phi * wv) @ phi.T
    F8 = ozaki.quadrature(phi, wv, g.becke, g.weights)
    assert np.array_equal(F8, F8.T)
    assert np.abs(F8 - F64).max() <= 1e-8 * np.abs(F64).max()
    E64 = 0.5 * (F64 * D).sum()
    assert abs(0.5 * (F8 * D).sum() - E64) <= 1e-8


def test_scheme_density_accuracy(h2o_case):
    import ozaki
    g, phi, D, rho, v = h2o_case
    r8 = ozaki.density(phi, D)
    assert np.abs(r8 - rho).max() <= 1e-7 * np.abs(rho).max()
    assert abs(g.integrate(r8) - g.integrate(rho)) <= 1e-8


def test_screened_scheme_matches_fp64(h2o_case):
    """The int8 mode's point screening: the dropped points carry
    |wb w| max phi^2 < 1e-24, so the screened quadrature and the screened
    density's integral match the full FP64 ones as closely as the unscreened
    scheme does."""
    import ozaki
    g, phi, D, rho, v = h2o_case
    keep = ozaki.screen(phi, g.becke, g.weights)
    mx = np.abs(phi).max(axis=0)
    assert np.array_equal(keep, (np.abs(g.becke * g.weights) * mx) * mx >= 1e-24)
    assert 0 < keep.sum() < keep.size       # this grid has points to drop
    wv = g.becke * g.weights * v
    F64 = (phi * wv) @ phi.T
    F8 = ozaki.quadrature(phi[:, keep], wv[keep], g.becke[keep], g.weights[keep])
    assert np.abs(F8 - F64).max() <= 1e-8 * np.abs(F64).max()
    r8 = np.zeros_like(rho)
    r8[keep] = ozaki.density(phi[:, keep], D)
    assert abs(g.integrate(r8) - g.integrate(rho)) <= 1e-8
    assert np.abs(g.becke * g.weights * rho)[~keep].sum() <= 1e-20
