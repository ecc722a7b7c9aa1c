"""Moving a grid, a basis and a Fock plan to a new geometry in place.

napmo_grid_set_centers rebuilds the atomic grid points around the new centres
with the expression of their construction, so the moved grid must equal a
grid built at the new geometry bit for bit (points, Becke weights, weights);
napmo_basis_set_origins + napmo_fock_plan_refresh must give the basis values
of a plan built from scratch.  GridChargeEnergy reuses one set of objects
across geometries; its energies, quadrature matrices and gradients must equal
those of fresh objects, also when forwards and gradients interleave.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

SYM = ['O', 'H', 'H']
R0 = np.array([(0.0, 0.0, 0.0), (0.0, 1.43, 1.11), (0.0, -1.43, 1.11)])


def _geoms(n, seed=5):
    rng = np.random.default_rng(seed)
    return [R0 + rng.uniform(-0.1, 0.1, size=R0.shape) for _ in range(n)]


def _system(R):
    from napmo_b200.system import MolecularSystem
    ms = MolecularSystem()
    for s, xyz in zip(SYM, R):
        ms.add_atom(s, xyz, units='BOHR', basis_name='CC-PVDZ')
    return ms


def test_moved_grid_equals_fresh_grid():
    import napmo_b200 as nb
    R1, R2 = _geoms(2)
    g = nb.BeckeGrid(_system(R1)['e-'], 40, 110)
    g.set_centers(R2)
    f = nb.BeckeGrid(_system(R2)['e-'], 40, 110)
    assert np.array_equal(g.points, f.points)
    assert np.array_equal(g.weights, f.weights)
    assert np.array_equal(g.becke_weights, f.becke_weights)


def test_moved_basis_and_refreshed_plan_equal_fresh_plan():
    import napmo_b200 as nb
    R1, R2 = _geoms(2, seed=9)
    e1 = _system(R1)['e-']
    g = nb.BeckeGrid(e1, 40, 110)
    fb = nb.FockBuilder(g, e1['basis'], 6)
    org = e1['basis'].origins()
    centre = [int(np.flatnonzero((R1 == o).all(axis=1))[0]) for o in org]
    g.set_centers(R2)
    e1['basis'].set_origins(R2[centre])
    fb.refresh()
    e2 = _system(R2)['e-']
    g2 = nb.BeckeGrid(e2, 40, 110)
    fb2 = nb.FockBuilder(g2, e2['basis'], 6)
    assert np.array_equal(e1['basis'].origins(), e2['basis'].origins())
    assert np.array_equal(fb.phi().cpu().numpy(), fb2.phi().cpu().numpy())
    n = fb.n
    rng = np.random.default_rng(3)
    C = rng.normal(size=(n, 5)) / np.sqrt(n)
    D = 2.0 * C @ C.T
    F1, rho1, v1 = fb.build(D)
    F2, rho2, v2 = fb2.build(D)
    assert np.array_equal(rho1.cpu().numpy(), rho2.cpu().numpy())
    assert np.array_equal(v1.cpu().numpy(), v2.cpu().numpy())
    assert np.array_equal(F1.cpu().numpy(), F2.cpu().numpy())


@pytest.mark.parametrize('species', ['e-', 'H_1'])
def test_grid_charge_energy_reuse_matches_fresh_objects(species):
    from napmo_b200.gradients import GridChargeEnergy
    kw = dict(species=species, quantum=(1, 2), nrad=40, nang=110)
    live = GridChargeEnergy(SYM, reuse=True, **kw)
    fresh = GridChargeEnergy(SYM, reuse=False, **kw)
    geoms = _geoms(3, seed=11)
    V0, _ = fresh.quadrature_matrix(geoms[0])
    n = V0.shape[0]
    rng = np.random.default_rng(n)
    C = rng.normal(size=(n, 2)) / np.sqrt(n)
    D = C @ C.T
    states = []
    for R in geoms:
        Va, sa = live.quadrature_matrix(R)
        Vb, sb = fresh.quadrature_matrix(R)
        assert np.array_equal(Va.cpu().numpy(), Vb.cpu().numpy())
        states.append((sa, sb))
    # gradients after all forwards: the live objects move back to each state
    for sa, sb in states:
        Ea, ga = live.gradient(sa, D)
        Eb, gb = fresh.gradient(sb, D)
        assert Ea == Eb
        assert np.array_equal(ga, gb)


def test_grid_charge_energy_int8_quadrature_matrix():
    """precision='int8x4': V = dE/dD from the int8 tensor-core quadrature
    (also after moves, which rebuild the int8 images) within 1e-8 of max|V| of
    the FP64 one; the gradient kernel is FP64 in both modes."""
    from napmo_b200.gradients import GridChargeEnergy
    kw = dict(species='e-', quantum=(1, 2), nrad=40, nang=110)
    m64 = GridChargeEnergy(SYM, **kw)
    m8 = GridChargeEnergy(SYM, precision='int8x4', **kw)
    for R in _geoms(2, seed=13):
        V, st = m64.quadrature_matrix(R)
        V8, st8 = m8.quadrature_matrix(R)
        V, V8 = V.cpu().numpy(), V8.cpu().numpy()
        assert np.abs(V8 - V).max() <= 1e-8 * np.abs(V).max()
        assert st8['fb'].tc_status() == 0


def test_screened_pair_lists_follow_their_mask():
    """Two int8 plans on one grid screen different points (different bases);
    the grid's Poisson plan keeps one set of screened pair lists and must
    rebuild it for the second plan's mask (keyed by the plan, not by the
    mask's address, which a freed plan's successor may reuse)."""
    import torch
    import napmo_b200 as nb
    from napmo_b200.system import MolecularSystem

    def system(basis):
        ms = MolecularSystem()
        for s, xyz in zip(SYM, R0):
            ms.add_atom(s, xyz, units='BOHR', basis_name=basis)
        return ms['e-']

    eA, eB, eB2 = system('CC-PVDZ'), system('STO-3G'), system('STO-3G')
    g = nb.BeckeGrid(eA, 40, 110)
    fA = nb.FockBuilder(g, eA['basis'], 6, precision='int8x4')
    DA = np.eye(fA.n) * 0.2
    fA.coulomb_potential(fA.density(DA))
    keepA = fA.kept_points()
    del fA
    fB = nb.FockBuilder(g, eB['basis'], 6, precision='int8x4')
    g2 = nb.BeckeGrid(eB2, 40, 110)
    fB2 = nb.FockBuilder(g2, eB2['basis'], 6, precision='int8x4')
    assert not torch.equal(keepA, fB.kept_points())
    DB = np.eye(fB.n) * 0.3
    vB = fB.coulomb_potential(fB.density(DB))
    vB2 = fB2.coulomb_potential(fB2.density(DB))
    assert torch.equal(vB, vB2)
