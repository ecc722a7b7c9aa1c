"""Int8-slice tensor-core contractions (tcgen05 kind::i8) on the GPU.

Two checks per result: (1) the kernels compute exactly the scheme restated in
oracle/ozaki.py (integer parts exact; only the order of the final FP64 sums
differs, so agreement to 1e-12 relative), and (2) the scheme's distance from
the FP64 path: rho within 1e-7 of max|rho|, F within 1e-8 of max|F|, and the
Fock-build energy 1/2 tr(D F) within 1e-6 Eh.
"""
import numpy as np
import pytest

from conftest import gpu_available
from helpers import H2O, product_system, random_density

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

BUTANE = [('C', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 1.54)), ('C', (0.0, 1.45, 2.05)),
          ('C', (0.0, 1.45, 3.59)), ('H', (1.03, 0.0, -0.36)), ('H', (-1.03, 0.0, -0.36)),
          ('H', (0.0, -1.03, -0.36)), ('H', (1.03, -0.5, 1.9)), ('H', (-1.03, -0.5, 1.9)),
          ('H', (1.03, 1.95, 1.7)), ('H', (-1.03, 1.95, 1.7)), ('H', (1.03, 0.95, 3.95)),
          ('H', (-1.03, 0.95, 3.95)), ('H', (0.0, 2.48, 3.95))]


def _phi_host(fb):
    return fb.phi().cpu().numpy()[:, :fb.npoint].copy()


@pytest.mark.parametrize('atoms,nrad,nang', [(H2O, 50, 110), (BUTANE, 40, 110)])
def test_int8_matches_scheme_and_fp64(atoms, nrad, nang):
    import napmo_b200 as nb
    import ozaki
    ms, grid = product_system(atoms, nrad=nrad, nang=nang)
    basis = ms['e-']['basis']
    n = basis['nbasis']
    D = random_density(n, ms['e-']['occupation'])
    rng = np.random.default_rng(7)
    v = 1.0 + rng.random(grid.size)
    f64 = nb.FockBuilder(grid, basis, -1)
    tc = nb.FockBuilder(grid, basis, -1, precision='int8x4')
    phi = _phi_host(f64)
    r64 = f64.density(D).cpu().numpy()
    r8 = tc.density(D).cpu().numpy()
    assert tc.tc_status() == 0
    rs = ozaki.density(phi, D)
    assert np.abs(r8 - rs).max() <= 1e-12 * np.abs(rs).max()
    assert np.abs(r8 - r64).max() <= 1e-7 * np.abs(r64).max()

    wb, w = grid.becke_weights, grid.weights
    F64 = f64.quadrature(1.0, v).cpu().numpy()
    F8 = tc.quadrature(1.0, v).cpu().numpy()
    assert tc.tc_status() == 0
    assert np.array_equal(F8, F8.T)
    Fs = ozaki.quadrature(phi, (wb * w) * v, wb, w)
    assert np.abs(F8 - Fs).max() <= 1e-12 * np.abs(Fs).max()
    assert np.abs(F8 - F64).max() <= 1e-8 * np.abs(F64).max()
    # determinism: same bits on a second call
    assert np.array_equal(F8, tc.quadrature(1.0, v).cpu().numpy())
    assert np.array_equal(r8, tc.density(D).cpu().numpy())


def test_int8_uneven_grid_and_signed_potential():
    """Per-atom grid sizes differ, the potential changes sign, n is not a
    multiple of any tile."""
    import napmo_b200 as nb
    import ozaki
    from napmo_b200.system import build_system
    ms = build_system(H2O, 'CC-PVDZ')
    grid = nb.BeckeGrid(ms['e-'], [40, 30, 30], [110, 50, 86])
    basis = ms['e-']['basis']
    rng = np.random.default_rng(11)
    v = rng.normal(size=grid.size)
    tc = nb.FockBuilder(grid, basis, -1, precision='int8x4')
    f64 = nb.FockBuilder(grid, basis, -1)
    F8 = tc.quadrature(1.0, v).cpu().numpy()
    F64 = f64.quadrature(1.0, v).cpu().numpy()
    wb, w = grid.becke_weights, grid.weights
    Fs = ozaki.quadrature(_phi_host(f64), (wb * w) * v, wb, w)
    assert tc.tc_status() == 0
    assert np.abs(F8 - Fs).max() <= 1e-12 * np.abs(Fs).max()
    assert np.abs(F8 - F64).max() <= 1e-8 * np.abs(F64).max()


@pytest.mark.parametrize('atoms,nrad,nang,nocc', [(H2O, 50, 110, 5), (BUTANE, 40, 110, 17)])
def test_int8_fock_build_energy(atoms, nrad, nang, nocc):
    import napmo_b200 as nb
    ms, grid = product_system(atoms, nrad=nrad, nang=nang)
    basis = ms['e-']['basis']
    D = random_density(basis['nbasis'], nocc)
    F64, rho64, _ = nb.FockBuilder(grid, basis, 8).build(D)
    tc = nb.FockBuilder(grid, basis, 8, precision='int8x4')
    F8, rho8, _ = tc.build(D)
    assert tc.tc_status() == 0
    E64 = 0.5 * float((F64.cpu().numpy() * D).sum())
    E8 = 0.5 * float((F8.cpu().numpy() * D).sum())
    assert abs(E64 - E8) <= 1e-6
    n64 = grid.integrate(rho64.cpu().numpy())
    n8 = grid.integrate(rho8.cpu().numpy())
    assert abs(n64 - n8) <= 1e-7
