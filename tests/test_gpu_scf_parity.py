"""Parity of the device SCF drivers with the oracle's grid SCF at the two SCF
configurations, and of one two-species Fock build at the APMO size.

  C1  GridRHF, H2O/cc-pVDZ, 50 x 110, grid J and orbital-pair exchange;
  C2  GridAPMO, HCN with a quantum H (5s5p), 100 x 302.

The converged oracle energies, iteration counts and densities come from
tests/golden/scf_oracle.json / .npz (tests/golden/make_scf_golden.py runs
oracle/scf.py, which restates the drivers on nAPMO's host arithmetic).  The
device must converge within 1e-8 Eh of the oracle in the same number of
iterations (+-1).  The build test runs the oracle live: rho, V_H and F of both
species from the oracle's converged densities, F within 1e-10 elementwise
(absolute) and 1e-10 of max|F|.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, gpu_available
from helpers import H2O, HCN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

E_TOL = 1e-8         # Eh, total energy against the oracle
F_TOL = 1e-10        # elementwise, Fock matrices against the oracle


def _golden():
    with open(os.path.join(GOLDEN, 'scf_oracle.json')) as f:
        return json.load(f), np.load(os.path.join(GOLDEN, 'scf_oracle.npz'))


def test_c1_rhf_converges_to_the_oracle_energy():
    from napmo_b200.scf import GridRHF
    from napmo_b200.system import build_system
    ref, _ = _golden()
    ref = ref['c1']
    res = GridRHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange='hf').run(tol=ref['tol'])
    assert res['converged'] and ref['converged']
    assert abs(res['energy'] - ref['energy']) <= E_TOL, (res['energy'], ref['energy'])
    assert abs(res['iterations'] - ref['iterations']) <= 1
    # the energies of the first iterations follow the oracle's path
    for (e_dev, _), (e_ref, _) in zip(res['history'][:4], ref['history'][:4]):
        assert abs(e_dev - e_ref) <= 1e-9


def test_c2_apmo_converges_to_the_oracle_energy():
    from napmo_b200.scf import GridAPMO
    from napmo_b200.system import build_system
    ref, _ = _golden()
    ref = ref['c2']
    ms = build_system(HCN, 'CC-PVDZ', quantum=(0,))
    res = GridAPMO(ms, 'H_1', 100, 302).run(tol=ref['tol'])
    assert res['converged'] and ref['converged']
    assert abs(res['energy'] - ref['energy']) <= E_TOL, (res['energy'], ref['energy'])
    assert abs(res['iterations'] - ref['iterations']) <= 1
    assert abs(res['electrons'] - 14.0) < 1e-8 and abs(res['nuclei'] - 1.0) < 1e-8


def test_c2_two_species_build_matches_the_oracle(oracle, basis_library, elements):
    """One coupled build at 100 x 302 from the oracle's converged densities:
    rho_e, rho_n, V[rho_e], V[rho_n] and the Coulomb + coupling parts of F_e
    (q_e^2 J[rho_e] + q_e q_n J[rho_n]) and F_n (q_n q_e J[rho_e])."""
    import scf as OS
    import torch
    from napmo_b200.scf import GridAPMO
    from napmo_b200.system import build_system
    _, arr = _golden()
    De, Dn = arr['c2_De'], arr['c2_Dn']
    ap = GridAPMO(build_system(HCN, 'CC-PVDZ', quantum=(0,)), 'H_1', 100, 302)
    e, n = ap.e, ap.nuc
    qq = e.q * n.q
    rho_e = e.fb.density(De)
    rho_n = n.fb.density(Dn)
    v_e = e.fb.coulomb_potential(rho_e)
    v_n = e.fb.coulomb_potential(rho_n)
    Fe = e.fb.quadrature(e.q * e.q, v_e, vext=qq * v_n)
    Fn = n.fb.quadrature(qq, v_e)
    torch.cuda.synchronize()
    orc = OS.GridAPMO(HCN, basis_library, elements, (0,), 100, 302)
    g = orc.grid
    assert np.array_equal(ap.grid.becke_weights, g.becke)
    r_e = oracle.density(orc.e.phi, De)
    r_n = oracle.density(orc.nuc.phi, Dn)
    V = OS.poisson_many(orc.plan, np.stack([r_e, r_n]))
    Fe_ref = oracle.quadrature(orc.e.phi, e.q * e.q * V[0] + qq * V[1], g.becke, g.weights)
    Fn_ref = oracle.quadrature(orc.nuc.phi, qq * V[0], g.becke, g.weights)
    checks = [(rho_e, r_e, 1e-12), (rho_n, r_n, 1e-12), (v_e, V[0], 1e-10), (v_n, V[1], 1e-10)]
    for dev, ref, tol in checks:
        dev = dev.cpu().numpy()
        assert np.abs(dev - ref).max() <= tol * np.abs(ref).max()
    for dev, ref in ((Fe, Fe_ref), (Fn, Fn_ref)):
        dev = dev.cpu().numpy()
        assert np.abs(dev - ref).max() <= F_TOL
        assert np.abs(dev - ref).max() <= F_TOL * np.abs(ref).max()
