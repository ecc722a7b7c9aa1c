"""Truncated multipole evaluation of the Poisson potential on the GPU.

With a tolerance tol > 0 every (atom, radial interval) bucket skips its
highest l-blocks whose Cauchy-Schwarz bound (Racah-normalised harmonics,
sum_m S_lm^2 = 1) sums to at most tol, so each point's potential moves by at
most natom * tol.  Checks: tol = 0 reproduces the full evaluation bit for bit
(it is the same code path as nAPMO's full sum), the bound holds for several
tolerances on a molecule and a random (non-physical) density, the truncated
potential is deterministic, and the precision modes set the tolerance (the
int8 mode also screens points: its potential is 0 at the dropped ones).
"""
import numpy as np
import pytest

from conftest import gpu_available
from helpers import H2O, product_system, random_density

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

PROPANE = [('C', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 1.54)), ('C', (0.0, 1.45, 2.05)),
           ('H', (1.03, 0.0, -0.36)), ('H', (-1.03, 0.0, -0.36)), ('H', (0.0, -1.03, -0.36)),
           ('H', (1.03, -0.5, 1.9)), ('H', (-1.03, -0.5, 1.9)), ('H', (1.03, 1.95, 1.7)),
           ('H', (-1.03, 1.95, 1.7)), ('H', (0.0, 2.48, 2.45))]


@pytest.mark.parametrize('atoms,nrad,nang,lmax', [(H2O, 50, 110, 8), (PROPANE, 40, 194, 11)])
def test_truncation_bound(atoms, nrad, nang, lmax):
    import torch
    import napmo_b200 as nb
    ms, grid = product_system(atoms, nrad=nrad, nang=nang)
    basis = ms['e-']['basis']
    D = random_density(basis['nbasis'], ms['e-']['occupation'])
    fb = nb.FockBuilder(grid, basis, lmax)
    rho = fb.density(D)
    v_ref = torch.empty_like(rho)
    nb.grids.coulomb_potential_device(grid, rho, lmax, v_ref)
    fb.set_poisson_tolerance(0.0)
    v0 = fb.coulomb_potential(rho)
    assert torch.equal(v0, v_ref)
    natom = len(atoms)
    for tol in (1e-12, 1e-10, 1e-8, 1e-6):
        fb.set_poisson_tolerance(tol)
        v = fb.coulomb_potential(rho)
        dv = float((v - v0).abs().max())
        assert dv <= natom * tol, (tol, dv)
        if tol == 1e-6:
            assert dv > 0.0  # some l-blocks were skipped
        assert torch.equal(v, fb.coulomb_potential(rho))


def test_precision_modes_set_the_tolerance():
    import torch
    import napmo_b200 as nb
    ms, grid = product_system(H2O, nrad=50, nang=110)
    basis = ms['e-']['basis']
    D = random_density(basis['nbasis'], 5)
    fb = nb.FockBuilder(grid, basis, 8)
    rho = fb.density(D)
    v0 = fb.coulomb_potential(rho)
    fb.set_precision('int8x4')
    keep = fb.kept_points()          # the int8 mode also screens points
    v8 = fb.coulomb_potential(rho)
    fb.set_poisson_tolerance(1e-9)         # the int8 mode's default
    assert torch.equal(v8, fb.coulomb_potential(rho))
    assert float((v8 - v0)[keep].abs().max()) <= 3 * 1e-9
    assert bool((v8[~keep] == 0.0).all())
    fb.set_precision('fp64')
    assert torch.equal(v0, fb.coulomb_potential(rho))
    fb.set_precision('int8x4', poisson_tol=0.0)
    v8 = fb.coulomb_potential(rho)
    assert torch.equal(v0[keep], v8[keep])
    with pytest.raises(nb.NapmoError):
        fb.set_poisson_tolerance(-1.0)
