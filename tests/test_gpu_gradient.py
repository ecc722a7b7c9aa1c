"""dE/dD and dE/dR of the grid quadrature energy E(D, R) of a species in the
potential of the classical nuclei (napmo_b200.gradients), checked against
central finite differences of the forward (step 1e-4 bohr), the forward's
own quadrature, and the CPU oracle's energy."""
import numpy as np
import pytest

from conftest import gpu_available
from helpers import BOHR, H2O, random_density

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

R0 = np.array([xyz for _, xyz in H2O]) / BOHR
SYM = [s for s, _ in H2O]


def _fd(model, D, R, h=1e-4):
    g = np.zeros_like(R)
    for a in range(R.shape[0]):
        for k in range(3):
            Rp, Rm = R.copy(), R.copy()
            Rp[a, k] += h
            Rm[a, k] -= h
            Ep = float((D * model.quadrature_matrix(Rp)[0].cpu().numpy()).sum())
            Em = float((D * model.quadrature_matrix(Rm)[0].cpu().numpy()).sum())
            g[a, k] = (Ep - Em) / (2 * h)
    return g


@pytest.mark.parametrize('species,quantum', [('e-', ()), ('H_1', (1, 2))])
@pytest.mark.parametrize('nrad,nang', [(30, 110), (75, 194)])
def test_gradient_matches_finite_differences(species, quantum, nrad, nang):
    """(75, 194) is the grid of the two-quantum-proton H2O configuration."""
    from napmo_b200.gradients import GridChargeEnergy
    model = GridChargeEnergy(SYM, species=species, quantum=quantum, nrad=nrad, nang=nang)
    R = R0 + np.random.default_rng(3).uniform(-0.05, 0.05, size=R0.shape) / BOHR
    V, state = model.quadrature_matrix(R)
    n = V.shape[0]
    D = random_density(n, 5 if species == 'e-' else 2, seed=17)
    E, g = model.gradient(state, D)
    E_fwd = float((D * V.cpu().numpy()).sum())
    assert abs(E - E_fwd) <= 1e-11 * abs(E_fwd)
    gfd = _fd(model, D, R)
    assert np.abs(g - gfd).max() <= 2e-6 * max(1.0, np.abs(gfd).max())
    # translation invariance: the total force on the system vanishes
    assert np.abs(g.sum(axis=0)).max() <= 1e-8 * max(1.0, np.abs(g).max())


def test_autograd_function():
    import torch
    from napmo_b200.gradients import GridChargeEnergy
    model = GridChargeEnergy(SYM, nrad=30, nang=110)
    V, state = model.quadrature_matrix(R0)
    D = torch.tensor(random_density(V.shape[0], 5, seed=2), dtype=torch.float64,
                     requires_grad=True)
    R = torch.tensor(R0, dtype=torch.float64, requires_grad=True)
    E = model(D, R)
    E.backward()
    _, g = model.gradient(state, D.detach().numpy())
    assert np.allclose(D.grad.numpy(), V.cpu().numpy(), rtol=0, atol=1e-14)
    assert np.allclose(R.grad.numpy(), g, rtol=1e-12, atol=1e-13)


def test_forward_matches_oracle(oracle, basis_library, elements):
    from helpers import oracle_system
    from napmo_b200.gradients import GridChargeEnergy
    model = GridChargeEnergy(SYM, nrad=30, nang=110)
    V, state = model.quadrature_matrix(R0)
    D = random_density(V.shape[0], 5, seed=9)
    E = float((D * V.cpu().numpy()).sum())
    g, fb = oracle_system(oracle, basis_library, elements, H2O, nrad=30, nang=110)
    phi = oracle.basis_compute(fb, g.points).T.copy()
    Z = {'O': 8, 'H': 1}
    v = np.zeros(g.size)
    for s, c in zip(SYM, R0):
        v -= Z[s] / np.linalg.norm(g.points - c, axis=1)
    Eo = float((D * oracle.quadrature(phi, v, g.becke, g.weights)).sum())
    assert abs(E - Eo) <= 1e-10 * abs(Eo)
