"""The oracle pinned against nAPMO's own known answers and against outputs of
nAPMO's compiled sources (tests/golden)."""
import numpy as np
import pytest

BOHR = 0.52917724924


def test_known_answer_basis_value(oracle, basis_library, known):
    # napmo/gto/test/test_basis_set.py: H STO-3G at the origin
    fb = oracle.flat_basis([[0.0, 0.0, 0.0]], ['H'], basis_library, 'STO-3G')
    phi = oracle.basis_compute(fb, np.zeros((1, 3)))
    np.testing.assert_allclose(phi[0, 0], known['basis_H_sto3g_phi0'], rtol=1e-7)


def test_known_answer_primitive_norms(oracle, known):
    # napmo/gto/test/test_primitive_gaussian.py
    np.testing.assert_allclose(oracle.lib.orc_prim_norm(np.zeros(3, np.int32), 0.5),
                               known['s_norm_zeta05'])
    np.testing.assert_allclose(oracle.lib.orc_prim_norm(np.array([0, 0, 3], np.int32), 0.5),
                               known['fz3_norm_zeta05'])
    fb = dict(l=np.array([0, 0, 3], np.int32), origin=np.zeros(3), nprim=np.array([1], np.int32),
              off=np.array([0], np.int32), zeta=np.array([0.5]), coeff=np.array([1.0]), nf=1)
    np.testing.assert_allclose(oracle.basis_compute(fb, np.ones((1, 3)))[0, 0],
                               known['fz3_value_at_111'])


def test_known_answer_radial_grid_he(oracle, elements, known):
    # napmo/wavefunction/test/test_kinetic.py: RadialGrid(50, 'He') points
    r, _ = oracle.radial_grid(50, elements['He']['atomic_radii'])
    np.testing.assert_allclose(r, known['radial_He_50_points'])


def test_known_answer_radial_integral(oracle):
    # napmo/grids/test/test_radial.py: int exp(-r^2/2) d3r = (2 pi)^1.5
    r, w = oracle.radial_grid(100, power=(0.0005, 1e1))
    assert abs(np.sum(np.exp(-0.5 * r ** 2) * w) - (2 * np.pi) ** 1.5) < 1e-9
    r, w = oracle.radial_grid(100, 0.5858151015155881)
    assert abs(np.sum(np.exp(-0.5 * r ** 2) * w) - (2 * np.pi) ** 1.5) < 1e-9


def test_known_answer_coulomb_h(oracle, basis_library, elements, known):
    # napmo/grids/test/test_coulomb.py: H STO-3G 1s^2 on 100 x 110, lmax 8
    g = oracle.Grid([[0.0, 0.0, 0.0]], [elements['H']['atomic_radii']], 100, 110)
    fb = oracle.flat_basis([[0.0, 0.0, 0.0]], ['H'], basis_library, 'STO-3G')
    phi = oracle.basis_compute(fb, g.points)[:, 0]
    rho = phi * phi
    v = oracle.compute_coulomb(g, rho, 8)
    assert np.allclose(g.integrate(rho * v), known['coulomb_H_sto3g_100x110'])


def test_spherical_average_h1s(oracle):
    # napmo/grids/test/test_spherical_average.py (decomposition of H 1s)
    atom = oracle.Atom(np.array([0.3, -0.2, 0.1]), 0.5858151015155881, 100, 110)
    d = np.sqrt(((atom.points - atom.center) ** 2).sum(axis=1))
    fn = np.exp(-2 * d) / np.pi
    sph = oracle.spherical_expansion(atom, fn, 4)
    check = np.exp(-2 * atom.r) / np.pi * np.sqrt(4 * np.pi)
    assert abs(sph[:, 0] - check).max() < 1e-10
    assert abs(sph[:, 1:]).max() < 1e-10


@pytest.mark.parametrize('order', [6, 14, 26, 38, 50, 74, 86, 110, 146, 170, 194, 230, 266,
                                   302, 350, 434, 590, 770, 974, 1202, 1454, 1730, 2030,
                                   2354, 2702, 3074, 3470, 3890, 4334, 4802, 5294, 5810])
def test_lebedev_bit_exact(oracle, refvec, order):
    pts, w = oracle.lebedev(order)
    ref = refvec['lebedev_%d' % order]
    assert np.array_equal(pts, ref[:, :3])
    assert np.array_equal(w, ref[:, 3])


@pytest.mark.parametrize('name,radii,n', [('cheb_H_100', 0.5858151015155881, 100),
                                          ('cheb_O_50', 1.2472192483880264, 50),
                                          ('cheb_C_75', 1.4069648596390618, 75)])
def test_radial_transform_bit_exact(oracle, refvec, name, radii, n):
    ref = refvec['rt_' + name]
    t = np.arange(n, dtype=np.float64)
    got = np.array([[oracle.lib.orc_cheb_radius(radii, n, x), oracle.lib.orc_cheb_deriv(radii, n, x),
                     oracle.lib.orc_cheb_deriv2(radii, n, x), oracle.lib.orc_cheb_deriv3(radii, n, x)]
                    for x in t])
    assert np.array_equal(got, ref)


@pytest.mark.parametrize('tag,atoms', [
    ('h2o', [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 1.430522, 1.109257)),
             ('H', (0.0, -1.430522, 1.109257))]),
    ('hcn', [('H', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 2.014455)), ('N', (0.0, 0.0, 4.199027))])])
def test_basis_values_vs_reference(oracle, refvec, basis_library, tag, atoms):
    fb = oracle.flat_basis([a[1] for a in atoms], [a[0] for a in atoms], basis_library, 'CC-PVDZ')
    phi = oracle.basis_compute(fb, refvec['gto_%s_points' % tag])
    np.testing.assert_allclose(phi, refvec['gto_%s_phi' % tag], rtol=1e-14, atol=1e-300)


def test_spline_dt_bit_exact(oracle, refvec):
    dt = np.zeros(40)
    oracle.lib.orc_spline_dt(refvec['spline_y'], dt, 40)
    assert np.array_equal(dt, refvec['spline_dt'])


def test_build_ode2_bit_exact(oracle, refvec):
    n = 12
    bcs = np.array([0.3, np.nan, -0.7, np.nan])
    coeffs = np.zeros((2 * n, 2 * n))
    rhs = np.zeros(2 * n)
    oracle.lib.orc_build_ode2(refvec['ode_b'], refvec['ode_a'], refvec['ode_f'], bcs, coeffs,
                              rhs, n)
    assert np.array_equal(coeffs, refvec['ode_coeffs'])
    assert np.array_equal(rhs, refvec['ode_rhs'])


def test_eval_decomposition_vs_reference(oracle, refvec):
    radii, nrad, lmax = refvec['dec_radii']
    nrad, lmax = int(nrad), int(lmax)
    pts = refvec['dec_points']
    out = np.zeros(pts.shape[0])
    oracle.lib.orc_eval_decomposition(0, radii, 0.0, nrad, (lmax + 1) ** 2,
                                      np.ascontiguousarray(refvec['dec_y']),
                                      np.ascontiguousarray(refvec['dec_dt']),
                                      np.ascontiguousarray(refvec['dec_center']), pts.shape[0],
                                      np.ascontiguousarray(pts), out)
    np.testing.assert_allclose(out, refvec['dec_out'], rtol=1e-13, atol=1e-13)


def test_becke_partition_of_unity(oracle, elements):
    # sum over owners of the Becke cell functions at one point is one: the
    # weights of the same physical point seen from each atom add to 1
    centers = np.array([[0.0, 0.0, 0.0], [0.0, 1.43, 1.11], [0.0, -1.43, 1.11]])
    radii = [elements[s]['atomic_radii'] for s in ('O', 'H', 'H')]
    g = oracle.Grid(centers, radii, 20, 26)
    assert np.all(g.becke >= 0) and np.all(g.becke <= 1)
    # electron count of a normalised 1s Gaussian on the middle atom
    r = np.sqrt(((g.points - centers[0]) ** 2).sum(axis=1))
    a = 2.0
    f = (2 * a / np.pi) ** 1.5 * np.exp(-2 * a * r * r)
    assert abs(g.integrate(f) - 1.0) < 1e-3   # 20 x 26 grid: quadrature error


def test_density_and_quadrature_small(oracle):
    rng = np.random.default_rng(1)
    n, N = 7, 300
    phi = rng.normal(size=(n, N))
    D = rng.normal(size=(n, n))
    D = D + D.T
    rho = oracle.density(phi, D)
    np.testing.assert_allclose(rho, np.einsum('ip,ij,jp->p', phi, D, phi), rtol=1e-12)
    C, bw, w = rng.normal(size=N), rng.uniform(size=N), rng.uniform(size=N)
    F = oracle.quadrature(phi, C, bw, w)
    np.testing.assert_allclose(F, (phi * (C * bw * w)) @ phi.T, rtol=1e-12, atol=1e-12)
