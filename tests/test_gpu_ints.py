"""One-electron integrals on the device (ints.cu: napmo_gpu_one_body and
nAPMO's LibintInterface one-body calls) against the oracle (oracle/ints.py,
McMurchie-Davidson with the Boys function from scipy's 1F1), nAPMO's compiled
overlaps and the H2/STO-3G textbook values.  Tolerances: 1e-12 of the
largest entry against the oracle (FP64, another Boys evaluation), 1e-13
against nAPMO's overlaps."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, gpu_available
from helpers import BOHR, H2O, HCN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]


@pytest.fixture(scope='module')
def library():
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'basis.json')) as f:
        return json.load(f)


def _device(basis, charges):
    import torch
    from napmo_b200 import cext
    n = basis['nbasis']
    q = np.ascontiguousarray(np.array([[*np.asarray(R, float), Z] for Z, R in charges],
                                      dtype=np.float64).reshape(-1, 4))
    out = [torch.empty((n, n), dtype=torch.float64, device='cuda') for _ in range(3)]
    cext.checked(cext.lib.napmo_gpu_one_body(basis._this, q.shape[0], q.ctypes.data,
                                             *[o.data_ptr() for o in out],
                                             torch.cuda.current_stream().cuda_stream))
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize('atoms,basis_name', [(H2O, 'CC-PVDZ'), (HCN, 'CC-PVDZ'),
                                              (H2O, '6-311G'), (HCN, 'STO-3G')])
def test_one_body_matches_oracle(library, atoms, basis_name):
    import ints as I
    import oracle as O
    from napmo_b200.system import build_system
    ms = build_system(atoms, basis_name)
    charges = [(pc['atomic_number'], pc['origin']) for pc in ms.point_charges]
    S, T, V = _device(ms['e-']['basis'], charges)
    cs = [np.array(x) / BOHR for _, x in atoms]
    fb = O.flat_basis(cs, [s for s, _ in atoms], library, basis_name)
    So, To, Vo = I.one_body(fb, [(Z, np.array(x) / BOHR) for (s, x), (Z, _) in
                                 zip(atoms, charges)])
    for dev, ref in ((S, So), (T, To), (V, Vo)):
        assert np.abs(dev - ref).max() <= 1e-12 * np.abs(ref).max()
        assert np.array_equal(dev, dev.T)


def test_overlap_matches_napmo_compiled(refvec):
    import napmo_b200 as nb
    atoms = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 1.430522, 1.109257)),
             ('H', (0.0, -1.430522, 1.109257))]
    from napmo_b200.system import build_system
    ms = build_system([(s, tuple(np.array(x) * BOHR)) for s, x in atoms], 'CC-PVDZ')
    S, _, _ = _device(ms['e-']['basis'], [])
    assert np.abs(S - refvec['ints_h2o_S']).max() <= 1e-13


def test_h2_sto3g_textbook():
    from napmo_b200.system import BOHR_TO_ANGSTROM, build_system
    ms = build_system([('H', (0.0, 0.0, 0.0)), ('H', (0.0, 0.0, 1.4 * BOHR_TO_ANGSTROM))],
                      'STO-3G')
    S, T, V = _device(ms['e-']['basis'], [(pc['atomic_number'], pc['origin'])
                                          for pc in ms.point_charges])
    H = T + V
    assert abs(S[0, 1] - 0.6593) < 5e-5 and abs(T[0, 0] - 0.7600) < 5e-5
    assert abs(H[0, 0] - (-1.1204)) < 5e-5 and abs(H[0, 1] - (-0.9584)) < 5e-5


def test_libint_interface_drop_in():
    """nAPMO's PSIA calls (psi_analytic.py:35-111): kinds 1, 2, 3 return the
    device S, T, V; an interface without charges returns V = 0."""
    from napmo_b200 import cext
    from napmo_b200.system import build_system
    ms = build_system(HCN, 'CC-PVDZ')
    b = ms['e-']['basis']
    charges = [(pc['atomic_number'], pc['origin']) for pc in ms.point_charges]
    S, T, V = _device(b, charges)
    lint = cext.lib.LibintInterface_new(0)
    cext.lib.LibintInterface_add_basis(lint, b._this)
    for Z, R in charges:
        cext.lib.LibintInterface_add_pointcharges(lint, int(Z), np.asarray(R, np.float64))
    n = cext.lib.LibintInterface_get_nbasis(lint)
    for kind, ref in ((1, S), (2, T), (3, V)):
        out = np.zeros((n, n))
        cext.lib.LibintInterface_compute_1body_ints(lint, kind, out)
        cext.check()
        assert np.array_equal(out, ref)
    cext.lib.LibintInterface_del(lint)
    lint = cext.lib.LibintInterface_new(0)
    cext.lib.LibintInterface_add_basis(lint, b._this)
    out = np.ones((n, n))
    cext.lib.LibintInterface_compute_1body_ints(lint, 3, out)
    assert not out.any()
    cext.lib.LibintInterface_del(lint)


def test_grid_rhf_with_analytic_hcore():
    """GridRHF with the device one-body integrals: V_ne equals the grid
    quadrature to the grid's accuracy (50 x 110: 1e-3 of max) and the SCF
    energy moves by the grid's V_ne error (measured 5.5e-4 Eh)."""
    from napmo_b200.scf import GridRHF
    from napmo_b200.system import build_system
    rg = GridRHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange='hf')
    ra = GridRHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange='hf', hcore='analytic')
    Vg, Va = rg.V.cpu().numpy(), ra.V.cpu().numpy()
    assert np.abs(Vg - Va).max() <= 1e-3 * np.abs(Va).max()
    Eg, Ea = rg.run(tol=1e-9)['energy'], ra.run(tol=1e-9)['energy']
    assert abs(Eg - Ea) < 1e-3


def test_f_functions_match_oracle():
    """s, p, d and f shells on two centres (the f instance of the kernel)
    against the oracle, with two point charges."""
    import ints as I
    from napmo_b200.gto import BasisSet
    shells = [(0, [2.0, 0.5], [0.4, 0.7]), (1, [0.9], [1.0]), (2, [0.8, 0.3], [0.5, 0.6]),
              (3, [1.2, 0.4], [0.6, 0.5])]
    centres = [np.array([0.1, -0.2, 0.3]), np.array([-0.4, 0.9, 1.6])]
    b = BasisSet('custom', 'X', centres[0], shells=shells)
    b.update(BasisSet('custom', 'X', centres[1], shells=shells))
    fb = dict(l=[], origin=[], nprim=[], off=[], zeta=[], coeff=[])
    for c in centres:
        for (lval, e, co) in shells:
            for k, i in enumerate(reversed(range(lval + 1))):
                for j in range(k + 1):
                    fb['l'] += [i, k - j, j]
                    fb['origin'] += list(c)
                    fb['off'].append(len(fb['zeta']))
                    fb['nprim'].append(len(e))
                    fb['zeta'] += list(e)
                    fb['coeff'] += list(co)
    fb = {k: np.array(v, np.int32 if k in ('l', 'nprim', 'off') else np.float64)
          for k, v in fb.items()}
    fb['nf'] = len(fb['nprim'])
    charges = [(3.0, centres[0]), (1.0, np.array([0.5, 0.5, -0.5]))]
    S, T, V = _device(b, charges)
    So, To, Vo = I.one_body(fb, charges)
    assert S.shape == (40, 40)
    for dev, ref in ((S, So), (T, To), (V, Vo)):
        assert np.abs(dev - ref).max() <= 1e-12 * np.abs(ref).max()


def test_many_charges_warp_kernel(library):
    """40 point charges (the warp-per-pair instance, used from 16 charges):
    V against the oracle to 1e-12 of its largest entry, S and T bit for bit
    those of the thread-per-pair instance."""
    import ints as I
    import oracle as O
    from napmo_b200.system import build_system
    ms = build_system(H2O, 'CC-PVDZ')
    rng = np.random.default_rng(11)
    charges = [(float(rng.uniform(0.1, 1.0)), rng.normal(scale=2.0, size=3)) for _ in range(40)]
    S, T, V = _device(ms['e-']['basis'], charges)
    S3, T3, _ = _device(ms['e-']['basis'], charges[:3])
    assert np.array_equal(S, S3) and np.array_equal(T, T3)
    cs = [np.array(x) / BOHR for _, x in H2O]
    fb = O.flat_basis(cs, [s for s, _ in H2O], library, 'CC-PVDZ')
    _, _, Vo = I.one_body(fb, charges)
    assert np.abs(V - Vo).max() <= 1e-12 * np.abs(Vo).max()
