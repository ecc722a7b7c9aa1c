"""Parity of the CUDA path (through libnapmo's C-ABI) with the oracle.

Tolerances: grid points, Becke weights and integer indices bit-exact; basis
values 1e-12 relative; F within 1e-10 of max|F| elementwise; potentials
within 1e-10 of max|v|; energies within 1e-8 Eh.
"""
import numpy as np
import pytest

from conftest import gpu_available
from helpers import H2O, HCN, BOHR, oracle_system, product_system, random_density

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]


@pytest.fixture(scope='module')
def h2o(oracle, basis_library, elements):
    ms, grid = product_system(H2O, nrad=50, nang=110)
    og, fb = oracle_system(oracle, basis_library, elements, H2O, nrad=50, nang=110)
    return ms, grid, og, fb


def test_grid_points_bit_exact(h2o):
    ms, grid, og, fb = h2o
    assert grid.size == og.size == 16500
    assert np.array_equal(grid.points, og.points)
    assert np.array_equal(grid.weights, og.weights)


def test_becke_weights_bit_exact_h2o(h2o):
    ms, grid, og, fb = h2o
    assert np.array_equal(grid.becke_weights, og.becke)


def test_becke_weights_bit_exact_uneven(oracle, basis_library, elements):
    import napmo_b200 as nb
    from napmo_b200.system import build_system
    ms = build_system(HCN)
    grid = nb.BeckeGrid(ms['e-'], [30, 40, 20], [110, 146, 194])
    centers = [np.array(xyz) / BOHR for _, xyz in HCN]
    radii = [elements[s]['atomic_radii'] for s, _ in HCN]
    og = oracle.Grid(centers, radii, [30, 40, 20], [110, 146, 194])
    assert np.array_equal(grid.points, og.points)
    assert np.array_equal(grid.becke_weights, og.becke)


def test_becke_weights_bit_exact_62_centres(oracle, elements):
    import napmo_b200 as nb
    from napmo_b200.system import alkane_geometry
    atoms = alkane_geometry()
    ms_species = dict(symbol='e-', particles=[dict(symbol=s, origin=np.array(x) / BOHR)
                                              for s, x in atoms])
    grid = nb.BeckeGrid(ms_species, 12, 26)
    og = oracle.Grid([np.array(x) / BOHR for _, x in atoms],
                     [elements[s]['atomic_radii'] for s, _ in atoms], 12, 26)
    assert np.array_equal(grid.becke_weights, og.becke)


@pytest.mark.parametrize('ncarbon', [66, 99])
def test_becke_weights_bit_exact_many_centres(oracle, elements, ncarbon):
    """200 and 299 centres: the centre tables no longer fit in shared memory
    (read from global memory; with and without the shared distance cache)."""
    import napmo_b200 as nb
    from napmo_b200.system import alkane_geometry
    atoms = alkane_geometry(ncarbon)
    assert len(atoms) in (200, 299)
    ms_species = dict(symbol='e-', particles=[dict(symbol=s, origin=np.array(x) / BOHR)
                                              for s, x in atoms])
    grid = nb.BeckeGrid(ms_species, 6, 14)
    og = oracle.Grid([np.array(x) / BOHR for _, x in atoms],
                     [elements[s]['atomic_radii'] for s, _ in atoms], 6, 14)
    assert np.array_equal(grid.becke_weights, og.becke)


def test_basis_values(h2o, oracle):
    ms, grid, og, fb = h2o
    pts = grid.points[::7]
    got = ms['e-']['basis'].compute(pts)
    ref = oracle.basis_compute(fb, pts)
    scale = np.abs(ref).max(axis=0)
    assert np.all(np.abs(got - ref) <= 1e-12 * scale + 1e-300)


def test_basis_values_vs_reference_vectors(refvec):
    import napmo_b200 as nb
    from napmo_b200.system import build_system
    atoms = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 1.430522, 1.109257)),
             ('H', (0.0, -1.430522, 1.109257))]
    ms = build_system([(s, tuple(np.array(x) * BOHR)) for s, x in atoms])
    got = ms['e-']['basis'].compute(refvec['gto_h2o_points'])
    ref = refvec['gto_h2o_phi']
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-16)


def test_basis_gradients_fd(h2o, oracle):
    ms, grid, og, fb = h2o
    pts = grid.points[::97]
    g = ms['e-']['basis'].deriv(pts)
    h = 1e-5
    for c in range(3):
        dp = np.zeros(3)
        dp[c] = h
        fd = (oracle.basis_compute(fb, pts + dp) - oracle.basis_compute(fb, pts - dp)) / (2 * h)
        assert np.abs(g[:, :, c] - fd).max() < 1e-6 * max(1.0, np.abs(fd).max())


def test_density(h2o, oracle):
    import napmo_b200 as nb
    ms, grid, og, fb = h2o
    basis = ms['e-']['basis']
    n = basis['nbasis']
    D = random_density(n, 5)
    fbld = nb.FockBuilder(grid, basis, 8)
    rho = fbld.density(D).cpu().numpy()
    phi = oracle.basis_compute(fb, og.points)
    ref = oracle.density(phi.T.copy(), D)
    assert np.abs(rho - ref).max() <= 1e-12 * np.abs(ref).max()


def test_quadrature_and_determinism(h2o, oracle):
    import napmo_b200 as nb
    ms, grid, og, fb = h2o
    basis = ms['e-']['basis']
    rng = np.random.default_rng(5)
    v = rng.normal(size=grid.size)
    fbld = nb.FockBuilder(grid, basis, -1)
    F1 = fbld.quadrature(1.0, v).cpu().numpy()
    F2 = fbld.quadrature(1.0, v).cpu().numpy()
    assert np.array_equal(F1, F2)
    assert np.array_equal(F1, F1.T)
    phi = oracle.basis_compute(fb, og.points)
    ref = oracle.quadrature(phi.T.copy(), v, og.becke, og.weights)
    assert np.abs(F1 - ref).max() <= 1e-10 * np.abs(ref).max()


def test_coulomb_known_answer(known, basis_library, elements, oracle):
    import napmo_b200 as nb
    ms = nb.MolecularSystem()
    ms.add_atom('H', [0.0, 0.0, 0.0], basis_name='STO-3G')
    grid = nb.BeckeGrid(ms['e-'], 100, 110)
    a = ms['e-']['basis']['cont'][0]
    rho = a.compute(grid.points) ** 2
    v = nb.compute_coulomb(grid, rho, 8)
    assert np.allclose(grid.integrate(rho * v), known['coulomb_H_sto3g_100x110'])
    og = oracle.Grid([[0.0, 0.0, 0.0]], [elements['H']['atomic_radii']], 100, 110)
    vref = oracle.compute_coulomb(og, rho, 8)
    assert np.abs(v - vref).max() <= 1e-10 * np.abs(vref).max()


@pytest.mark.parametrize('lmax', [2, 8])
def test_coulomb_h2o_vs_oracle(h2o, oracle, lmax):
    import napmo_b200 as nb
    ms, grid, og, fb = h2o
    phi = oracle.basis_compute(fb, og.points)
    D = random_density(phi.shape[1], 5)
    rho = oracle.density(phi.T.copy(), D)
    v = nb.compute_coulomb(grid, rho, lmax)
    vref = oracle.compute_coulomb(og, rho, lmax)
    assert np.abs(v - vref).max() <= 1e-10 * np.abs(vref).max()


def test_spherical_expansion(oracle, elements):
    import napmo_b200 as nb
    R = np.array([0.2, -0.1, 0.4])
    g = nb.AtomicGrid(60, 194, R, 'O')
    o = oracle.Atom(R, elements['O']['atomic_radii'], 60, 194)
    rng = np.random.default_rng(2)
    d = np.sqrt(((o.points - R) ** 2).sum(1))
    f = np.exp(-d) * (1 + o.points[:, 0] * o.points[:, 2]) + 0.01 * rng.normal(size=o.size)
    got = g.spherical_expansion(11, f)
    ref = oracle.spherical_expansion(o, f, 11)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize('nrad', [2, 3, 5, 17, 40])
def test_poisson_solver_splines(oracle, basis_library, elements, nrad):
    """Radial solutions against the oracle, down to radial grids shorter than
    the radial kernel's prefetch rings (the sweeps' prologues and tails)."""
    import napmo_b200 as nb
    atoms = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.757, 0.587))]
    ms, grid = product_system(atoms, nrad=nrad, nang=86)
    og, fb = oracle_system(oracle, basis_library, elements, atoms, nrad=nrad, nang=86)
    phi = oracle.basis_compute(fb, og.points)
    rho = oracle.density(phi.T.copy(), random_density(phi.shape[1], 4))
    U = nb.poisson_solver(grid, rho, 7)
    Uref = oracle.poisson_solver(og, rho, 7)
    for a in range(2):
        y = np.array([s.y for s in U[a]])
        dt = np.array([s.dt for s in U[a]])
        yr, dtr = Uref[a]
        assert np.abs(y - yr).max() <= 1e-10 * np.abs(yr).max()
        assert np.abs(dt - dtr).max() <= 1e-10 * np.abs(dtr).max()


def test_eval_decomposition_vs_reference(refvec):
    import napmo_b200 as nb
    radii, nrad, lmax = refvec['dec_radii']
    nrad, lmax = int(nrad), int(lmax)
    rt = nb.ChebyshevRadialTransform(radii, nrad)
    splines = []
    c = 0
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            y = np.ascontiguousarray(refvec['dec_y'][c])
            dt = np.ascontiguousarray(refvec['dec_dt'][c])
            splines.append(nb.CubicSpline(y, dt, rt, nb.PotentialExtrapolation(l), v=np.ones(nrad)))
            c += 1
    pts = np.ascontiguousarray(refvec['dec_points'])
    out = np.zeros(pts.shape[0])
    arr = np.array([s._this for s in splines], dtype=np.uintp).astype(object)
    from ctypes import c_void_p
    sp = np.array([s._this for s in splines], dtype=c_void_p)
    cell = nb.Cell(None)
    nb.cext.lib.eval_decomposition_grid(sp, np.ascontiguousarray(refvec['dec_center']), out, pts,
                                        cell._this, len(splines), pts.shape[0])
    nb.cext.check()
    np.testing.assert_allclose(out, refvec['dec_out'], rtol=1e-12, atol=1e-12)


def test_fock_build_end_to_end(h2o, oracle):
    import napmo_b200 as nb
    ms, grid, og, fb = h2o
    basis = ms['e-']['basis']
    n = basis['nbasis']
    D = random_density(n, 5)
    fbld = nb.FockBuilder(grid, basis, 8)
    F, rho, v = fbld.build(D)
    F = F.cpu().numpy()
    phi = oracle.basis_compute(fb, og.points)
    rho_ref = oracle.density(phi.T.copy(), D)
    v_ref = oracle.compute_coulomb(og, rho_ref, 8)
    F_ref = oracle.quadrature(phi.T.copy(), v_ref, og.becke, og.weights)
    assert np.abs(F - F_ref).max() <= 1e-10 * np.abs(F_ref).max()
    E, E_ref = 0.5 * np.sum(D * F), 0.5 * np.sum(D * F_ref)
    assert abs(E - E_ref) <= 1e-8
    # host-buffer path through the C-ABI gives the same matrix
    Fh = fbld.build_host(D)
    assert np.array_equal(Fh, F)


def test_legacy_coupling_entry_point(h2o, oracle):
    import napmo_b200 as nb
    from ctypes import byref
    ms, grid, og, fb = h2o
    basis = ms['e-']['basis']
    n = basis['nbasis']
    phi = np.ascontiguousarray(basis.compute(grid.points).T)
    rng = np.random.default_rng(9)
    J = rng.normal(size=grid.size)
    psi = nb.WaveFunction(n, 5)
    res = np.zeros((n, n))
    nb.cext.lib.nwavefunction_compute_coupling(byref(psi), grid._this, phi, J, res)
    nb.cext.check()
    ref = oracle.quadrature(phi, J, og.becke, og.weights)
    assert np.abs(res - ref).max() <= 1e-10 * np.abs(ref).max()


def test_scf_step_matches_eigh():
    import scipy.linalg
    import napmo_b200 as nb
    rng = np.random.default_rng(4)
    n = 12
    A = rng.normal(size=(n, n))
    S = A @ A.T / n + np.eye(n)
    F = rng.normal(size=(n, n))
    F = F + F.T
    psi = nb.WaveFunction(n, 3)
    psi.S[:] = S
    psi.F[:] = F
    psi.H[:] = np.eye(n)
    psi.iterate()
    w, C = scipy.linalg.eigh(F, S)
    np.testing.assert_allclose(psi.O, w, rtol=1e-10, atol=1e-12)
    D = 2.0 * C[:, :3] @ C[:, :3].T
    np.testing.assert_allclose(psi.D, D, rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(psi.energy, np.sum(D * np.eye(n)), rtol=1e-10)


def test_nuclear_potential(h2o, oracle):
    import napmo_b200 as nb
    ms, grid, og, fb = h2o
    v = nb.compute_nuclear(grid, ms.point_charges)
    ref = oracle.nuclear_potential(og.points, [(p['atomic_number'], p['origin'])
                                               for p in ms.point_charges])
    np.testing.assert_allclose(v, ref, rtol=1e-13)


def test_multigrid_common_points(known):
    import napmo_b200 as nb
    sp = {'symbol': 'e-', 'particles': [{'symbol': 'H', 'origin': np.array([0, 0, 0.6935])},
                                        {'symbol': 'H', 'origin': np.array([0, 0, -0.6935])}]}
    sp2 = {'symbol': 'H_1', 'particles': [{'symbol': 'H_1', 'origin': np.array([0, 0, -0.6935])}]}
    g1 = nb.BeckeGrid(sp, 50, 110)
    g2 = nb.BeckeGrid(sp2, 50, 110)
    mg = nb.MultiGrid(2)
    mg.add_grid(g1)
    mg.add_grid(g2)
    cp = mg.get_common_points('e-', 'H_1')
    assert cp.shape[0] == known['multigrid_common_points']
    assert np.array_equal(cp[:, 0], np.arange(5500, 11000))
    assert np.array_equal(cp[:, 1], np.arange(0, 5500))
