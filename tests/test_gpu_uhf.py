"""Unrestricted grid SCF (napmo_b200.scf.GridUHF / GridMultiSCF: nAPMO's
method 'uhf', electrons split into e-alpha and e-beta) against the oracle's
restatement (oracle/scf.py: GridMultiSCF), converged energies in
tests/golden/scf_oracle.json (tests/golden/make_scf_golden.py):

  * closed-shell H2O: the UHF equals the RHF energy of the C1 fixture;
  * OH radical (doublet), 50 x 110: energy within 1e-8 Eh, iterations +-1,
    5 alpha and 4 beta electrons;
  * OH radical with a quantum proton (APMO-UHF), 50 x 110;
  * neutral HCN with a quantum proton: APMO-UHF equals APMO-RHF;
  * spin-polarised LDA (unrestricted Kohn-Sham, nAPMO's DFT for open
    shells): OH radical within 1e-8 Eh of the oracle's, closed-shell H2O equal
    to the restricted LDA SCF, and the HF/DFT solver front end dispatching to it.
"""
import json
import os

import pytest

from conftest import GOLDEN, gpu_available
from helpers import H2O, HCN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

OH = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.0, 0.97))]
E_TOL = 1e-8


def _ref(case):
    with open(os.path.join(GOLDEN, 'scf_oracle.json')) as f:
        return json.load(f)[case]


def test_closed_shell_uhf_equals_rhf():
    from napmo_b200.scf import GridUHF
    from napmo_b200.system import build_system
    ref = _ref('c1')
    res = GridUHF(build_system(H2O, 'CC-PVDZ'), 50, 110).run(tol=ref['tol'])
    assert res['converged']
    assert abs(res['energy'] - ref['energy']) <= E_TOL
    assert abs(res['alpha'] - 5.0) < 1e-8 and abs(res['beta'] - 5.0) < 1e-8


def test_uhf_oh_radical_matches_the_oracle():
    from napmo_b200.scf import GridUHF
    from napmo_b200.system import build_system
    ref = _ref('uhf_oh')
    res = GridUHF(build_system(OH, 'CC-PVDZ'), 50, 110).run(tol=ref['tol'])
    assert res['converged'] and ref['converged']
    assert abs(res['energy'] - ref['energy']) <= E_TOL, (res['energy'], ref['energy'])
    assert abs(res['iterations'] - ref['iterations']) <= 1
    assert abs(res['alpha'] - 5.0) < 1e-8 and abs(res['beta'] - 4.0) < 1e-8


def test_apmo_uhf_oh_matches_the_oracle():
    from napmo_b200.scf import GridMultiSCF
    from napmo_b200.system import build_system
    ref = _ref('apmo_uhf_oh')
    ms = build_system(OH, 'CC-PVDZ', quantum=(1,))
    res = GridMultiSCF(ms, 'H_1', 50, 110).run(tol=ref['tol'])
    assert res['converged'] and ref['converged']
    assert abs(res['energy'] - ref['energy']) <= E_TOL, (res['energy'], ref['energy'])
    assert abs(res['iterations'] - ref['iterations']) <= 1
    assert abs(res['alpha'] - 5.0) < 1e-8 and abs(res['beta'] - 4.0) < 1e-8
    assert abs(res['nuclei'] - 1.0) < 1e-8


def test_closed_shell_apmo_uhf_equals_apmo_rhf():
    from napmo_b200.scf import GridAPMO, GridMultiSCF
    from napmo_b200.system import build_system
    r = GridAPMO(build_system(HCN, 'CC-PVDZ', quantum=(0,)), 'H_1', 50, 110).run(tol=1e-10)
    u = GridMultiSCF(build_system(HCN, 'CC-PVDZ', quantum=(0,)), 'H_1', 50, 110).run(tol=1e-10)
    assert r['converged'] and u['converged']
    assert abs(r['energy'] - u['energy']) <= 1e-8


def test_uks_oh_radical_matches_the_oracle():
    from napmo_b200.scf import GridUHF
    from napmo_b200.system import build_system
    ref = _ref('uks_oh')
    res = GridUHF(build_system(OH, 'CC-PVDZ'), 50, 110, exchange='lda').run(tol=ref['tol'])
    assert res['converged'] and ref['converged']
    assert abs(res['energy'] - ref['energy']) <= E_TOL, (res['energy'], ref['energy'])
    assert abs(res['iterations'] - ref['iterations']) <= 1
    assert abs(res['alpha'] - 5.0) < 1e-8 and abs(res['beta'] - 4.0) < 1e-8


def test_closed_shell_uks_equals_rks():
    from napmo_b200.scf import GridRHF, GridUHF
    from napmo_b200.system import build_system
    rks = GridRHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange='lda').run(tol=1e-9)
    uks = GridUHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange='lda').run(tol=1e-9)
    assert rks['converged'] and uks['converged']
    assert abs(uks['energy'] - rks['energy']) <= 1e-8, (uks['energy'], rks['energy'])


def test_dft_solver_open_shell_runs_polarised_lda():
    import napmo_b200 as nb
    from napmo_b200.system import build_system
    ref = _ref('uks_oh')
    ms = build_system(OH, 'CC-PVDZ')
    E = nb.DFT(ms, {'grid': [50, 110], 'eps_e': ref['tol']}).compute()
    assert abs(E - ref['energy']) <= E_TOL, (E, ref['energy'])
