"""Batched Poisson solves (napmo_gpu_poisson_many, napmo_fock_plan_poisson_many):
one launch per pipeline stage for k densities gives the same potentials, bit
for bit, as k single solves, untruncated and truncated, on the full and on a
screened (int8 plan) point set."""
import numpy as np
import pytest

from conftest import gpu_available
from helpers import H2O, product_system

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]


def _densities(torch, grid, k, seed=5):
    rng = np.random.default_rng(seed)
    pts = grid.points
    rows = []
    for j in range(k):
        c = rng.normal(scale=1.0, size=3)
        a = rng.uniform(0.3, 2.0)
        rows.append(np.exp(-a * ((pts - c) ** 2).sum(1)) * rng.normal())
    return torch.as_tensor(np.array(rows), device='cuda')


@pytest.mark.parametrize('tol', [0.0, 1e-10])
def test_grid_batch_equals_single(tol):
    import torch
    from napmo_b200 import cext
    from napmo_b200.grids import coulomb_potential_device
    ms, grid = product_system(H2O, nrad=50, nang=110)
    grid.set_poisson_tolerance(tol)
    rho = _densities(torch, grid, 7)
    N = grid.size
    V = torch.empty_like(rho)
    cext.checked(cext.lib.napmo_gpu_poisson_many(grid._this, 7, rho.data_ptr(), N, 8,
                                                 V.data_ptr(),
                                                 torch.cuda.current_stream().cuda_stream))
    for j in range(7):
        v = torch.empty(N, dtype=torch.float64, device='cuda')
        coulomb_potential_device(grid, rho[j].contiguous(), 8, v)
        assert torch.equal(v, V[j]), j


def test_plan_batch_equals_single_int8_screened():
    import torch
    import napmo_b200 as nb
    ms, grid = product_system(H2O, nrad=50, nang=110)
    fb = nb.FockBuilder(grid, ms['e-']['basis'], 8)
    fb.set_precision('int8x4')          # truncation 1e-10 and point screening
    rho = _densities(torch, grid, 5, seed=9)
    V = fb.coulomb_potentials(rho)
    for j in range(5):
        assert torch.equal(fb.coulomb_potential(rho[j]), V[j]), j
