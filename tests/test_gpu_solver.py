"""napmo_b200.HF / DFT: nAPMO's solver interface (hf_solver.py, dft_solver.py)
over the grid drivers.  Each solver's energy equals the driver it dispatches
to, and the oracle fixtures where they exist."""
import json
import os

import pytest

from conftest import GOLDEN, gpu_available
from helpers import H2O, HCN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

OH = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.0, 0.97))]


def _ref(case):
    with open(os.path.join(GOLDEN, 'scf_oracle.json')) as f:
        return json.load(f)[case]


def test_hf_rhf_and_uhf():
    import napmo_b200 as nb
    from napmo_b200.system import build_system
    ref = _ref('c1')
    E = nb.HF(build_system(H2O, 'CC-PVDZ'), {'grid': [50, 110], 'eps_e': ref['tol']},
              pprint=False).compute()
    assert abs(E - ref['energy']) <= 1e-8
    ref = _ref('uhf_oh')
    E = nb.HF(build_system(OH, 'CC-PVDZ'), {'grid': {'e-': {'nrad': 50, 'nang': 110}},
                                             'eps_e': ref['tol']}, pprint=False).compute()
    assert abs(E - ref['energy']) <= 1e-8


def test_hf_apmo_and_charged_open_shell():
    import napmo_b200 as nb
    from napmo_b200.scf import GridAPMO
    from napmo_b200.system import build_system
    solver = nb.HF(build_system(HCN, 'CC-PVDZ', quantum=(0,)), {'grid': [50, 110], 'eps_e': 1e-9},
                   pprint=False)
    E = solver.compute()
    assert isinstance(solver.driver, GridAPMO)
    E2 = GridAPMO(build_system(HCN, 'CC-PVDZ', quantum=(0,)), 'H_1', 50, 110).run(tol=1e-9)
    assert abs(E - E2['energy']) <= 1e-10
    ref = _ref('apmo_uhf_oh')
    E = nb.HF(build_system(OH, 'CC-PVDZ', quantum=(1,)), {'grid': [50, 110], 'method': 'uhf',
                                                          'eps_e': ref['tol']},
              pprint=False).compute()
    assert abs(E - ref['energy']) <= 1e-8
    # H2O+ (doublet) through set_charges: the open-shell driver at charge +1
    from napmo_b200.scf import GridUHF
    ms = build_system(H2O, 'CC-PVDZ').set_charges({'e-': {'charge': -1}})
    assert ms.open_shell
    solver = nb.HF(ms, {'grid': [50, 110], 'eps_e': 1e-9}, pprint=False)
    E = solver.compute()
    assert isinstance(solver.driver, GridUHF)
    r = GridUHF(build_system(H2O, 'CC-PVDZ'), 50, 110, charge=1).run(tol=1e-9)
    assert abs(E - r['energy']) <= 1e-10


def test_dft_lda_and_epc():
    import napmo_b200 as nb
    from napmo_b200.scf import GridAPMO, GridRHF
    from napmo_b200.system import build_system
    E = nb.DFT(build_system(H2O, 'CC-PVDZ'), {'grid': [50, 110], 'eps_e': 1e-9},
               pprint=False).compute()
    r = GridRHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange='lda').run(tol=1e-9)
    assert abs(E - r['energy']) <= 1e-10
    opts = {'grid': [50, 110], 'eps_e': 1e-9, 'functional': {'e-': 'lda', 'e-:H_1': 'epc17-2'}}
    E = nb.DFT(build_system(HCN, 'CC-PVDZ', quantum=(0,)), opts, pprint=False).compute()
    r = GridAPMO(build_system(HCN, 'CC-PVDZ', quantum=(0,)), 'H_1', 50, 110, exchange='lda',
                 correlation='epc17-2').run(tol=1e-9)
    assert abs(E - r['energy']) <= 1e-10
