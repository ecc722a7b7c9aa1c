"""Parity at the large single-system size: C20H42/cc-pVDZ (510 Cartesian
functions), 100 x 302 per atom, 62 atoms, 1,872,400 points.  The oracle cannot
redo the whole build in a test (phi alone is 7.6 GB), so it checks a seeded
sample of 4,096 grid points:

  * Becke weights of the sampled points, bit for bit (becke.cpp:79-176 per
    point with its owning atom);
  * phi at the sampled points (basis_set.cpp:69-82), 1e-12 of max;
  * rho at the sampled points from the sampled phi, 1e-12 of max;
  * V_H at the sampled points: the oracle's Poisson solve (projection of every
    atom's points, radial FEM solves, multipole evaluation at the sample) of
    the device density, 1e-10 of max.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

SEED = 20261203
NSAMPLE = 4096


def test_c20h42_sampled_points_match_the_oracle(oracle, basis_library, elements):
    import scf as OS
    import torch
    import napmo_b200 as nb
    from helpers import BOHR, random_density
    from napmo_b200.system import alkane_geometry, build_system
    atoms = alkane_geometry(20)
    ms = build_system(atoms, 'CC-PVDZ')
    grid = nb.BeckeGrid(ms['e-'], 100, 302)
    lmax = nb.lebedev_get_order(302) // 2
    fb = nb.FockBuilder(grid, ms['e-']['basis'], lmax)
    n, N = fb.n, grid.size
    assert (n, N) == (510, 1872400)
    D = random_density(n, 81, SEED)
    rho = fb.density(D)
    v = fb.coulomb_potential(rho)
    rng = np.random.default_rng(SEED)
    idx = np.sort(rng.choice(N, NSAMPLE, replace=False))
    phi_s = fb.phi()[:, torch.as_tensor(idx, device='cuda')].cpu().numpy()
    rho_d = rho.cpu().numpy()
    v_s = v.cpu().numpy()[idx]
    torch.cuda.synchronize()

    centers = [np.array(xyz, dtype=np.float64) / BOHR for _, xyz in atoms]
    radii = [elements[s]['atomic_radii'] for s, _ in atoms]
    og = oracle.Grid(centers, radii, 100, 302, becke=False)
    assert np.array_equal(grid.points, og.points)
    assert np.array_equal(grid.weights, og.weights)
    wb = og.becke_sample(idx)
    assert np.array_equal(grid.becke_weights[idx], wb)

    ofb = oracle.flat_basis(centers, [s for s, _ in atoms], basis_library, 'CC-PVDZ')
    phi_ref = oracle.basis_compute(ofb, og.points[idx]).T.copy()
    assert np.abs(phi_s - phi_ref).max() <= 1e-12 * np.abs(phi_ref).max()
    rho_ref = oracle.density(phi_ref, D)
    assert np.abs(rho_d[idx] - rho_ref).max() <= 1e-12 * np.abs(rho_ref).max()

    # the oracle's Poisson solve of the device density (Becke weights of the
    # whole grid from the device: the sampled ones are equal bit for bit)
    og.becke = np.ascontiguousarray(grid.becke_weights)
    plan = OS.PoissonPlan(og, lmax)
    v_ref = OS.poisson_many(plan, rho_d[None, :], points=og.points[idx])[0]
    assert np.abs(v_s - v_ref).max() <= 1e-10 * np.abs(v_ref).max()
