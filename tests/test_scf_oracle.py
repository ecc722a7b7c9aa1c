"""The oracle's grid SCF (oracle/scf.py) on the host: its batched Poisson
solve against the per-(l, m) restatement of poisson_solver.py, its sampled
evaluations and Becke weights against the whole-grid ones, and the C1 SCF
against the committed fixture (tests/golden/scf_oracle.json) that the GPU
tests compare the device drivers with."""
import json
import os

import numpy as np

from conftest import GOLDEN
from helpers import H2O, oracle_system, random_density


def _system(oracle, basis_library, elements, nrad=30, nang=50):
    g, fb = oracle_system(oracle, basis_library, elements, H2O, nrad=nrad, nang=nang)
    phi = oracle.basis_compute(fb, g.points).T.copy()
    return g, phi


def test_batched_poisson_equals_the_per_lm_solves(oracle, basis_library, elements):
    import scf as OS
    g, phi = _system(oracle, basis_library, elements)
    lmax = 5
    rho = oracle.density(phi, random_density(phi.shape[0], 5))
    dens = np.stack([rho, phi[0] * phi[3], phi[2] * phi[7]])
    V = OS.poisson_many(OS.PoissonPlan(g, lmax), dens)
    for k in range(3):
        ref = oracle.compute_coulomb(g, dens[k], lmax)
        assert np.abs(V[k] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_sampled_evaluation_and_becke_weights(oracle, basis_library, elements):
    import scf as OS
    g, phi = _system(oracle, basis_library, elements)
    plan = OS.PoissonPlan(g, 4)
    dens = np.stack([phi[1] * phi[1], phi[4] * phi[9]])
    V = OS.poisson_many(plan, dens)
    idx = np.sort(np.random.default_rng(3).choice(g.size, 300, replace=False))
    Vs = OS.poisson_many(plan, dens, points=g.points[idx])
    assert np.array_equal(Vs, V[:, idx])
    assert np.array_equal(g.becke_sample(idx), g.becke[idx])


def test_c1_scf_reproduces_the_fixture(basis_library, elements):
    import scf as OS
    with open(os.path.join(GOLDEN, 'scf_oracle.json')) as f:
        ref = json.load(f)['c1']
    res = OS.GridRHF(H2O, basis_library, elements, 50, 110).run(tol=ref['tol'])
    assert res['converged'] and res['iterations'] == ref['iterations']
    assert abs(res['energy'] - ref['energy']) <= 1e-10
    assert abs(res['electrons'] - 10.0) < 1e-10
    D = np.load(os.path.join(GOLDEN, 'scf_oracle.npz'))['c1_D']
    assert np.abs(res['D'] - D).max() <= 1e-8


def test_reference_arm_geometry_equals_the_product_one():
    """bench.py's host arm builds C20H42 without loading libnapmo.so."""
    import workloads
    from napmo_b200.system import alkane_geometry
    a, b = workloads.alkane_geometry(20), alkane_geometry(20)
    assert [s for s, _ in a] == [s for s, _ in b]
    assert np.array_equal(np.array([x for _, x in a]), np.array([x for _, x in b]))


def test_uks_scf_reproduces_the_fixture(basis_library, elements):
    """Spin-polarised LDA (unrestricted Kohn-Sham) of the OH radical: the
    oracle reproduces the committed fixture the GPU test compares with."""
    import scf as OS
    with open(os.path.join(GOLDEN, 'scf_oracle.json')) as f:
        ref = json.load(f)['uks_oh']
    oh = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.0, 0.97))]
    res = OS.GridMultiSCF(oh, basis_library, elements, (), 50, 110,
                          exchange='lda').run(tol=ref['tol'])
    assert res['converged'] and res['iterations'] == ref['iterations']
    assert abs(res['energy'] - ref['energy']) <= 1e-10
