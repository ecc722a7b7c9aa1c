"""One-electron integrals of the oracle (CPU): the H2/STO-3G values of
Szabo and Ostlund (Modern Quantum Chemistry, section 3.5.2), nAPMO's own
compiled contracted overlaps (tests/golden/reference_vectors.npz), and the
product's host overlap/kinetic matrices."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from helpers import BOHR, H2O, HCN


@pytest.fixture(scope='module')
def library():
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'basis.json')) as f:
        return json.load(f)


def test_oracle_h2_sto3g_textbook(library):
    import ints as I
    import oracle as O
    cs = [np.zeros(3), np.array([0.0, 0.0, 1.4])]
    fb = O.flat_basis(cs, ['H', 'H'], library, 'STO-3G')
    S, T, V = I.one_body(fb, [(1.0, cs[0]), (1.0, cs[1])])
    _, _, V1 = I.one_body(fb, [(1.0, cs[0])])
    H = T + V
    close = lambda a, b: abs(a - b) < 5e-5
    assert close(S[0, 1], 0.6593) and close(T[0, 0], 0.7600) and close(T[0, 1], 0.2365)
    assert close(V1[0, 0], -1.2266) and close(V1[0, 1], -0.5974) and close(V1[1, 1], -0.6538)
    assert close(H[0, 0], -1.1204) and close(H[0, 1], -0.9584)


@pytest.mark.parametrize('tag,atoms', [
    ('h2o', [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 1.430522, 1.109257)),
             ('H', (0.0, -1.430522, 1.109257))]),
    ('hcn', [('H', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 2.014455)), ('N', (0.0, 0.0, 4.199027))])])
def test_oracle_overlap_matches_napmo_compiled(library, refvec, tag, atoms):
    import ints as I
    import oracle as O
    fb = O.flat_basis([np.array(x) for _, x in atoms], [s for s, _ in atoms], library, 'CC-PVDZ')
    S, _, _ = I.one_body(fb, [])
    assert np.abs(S - refvec['ints_%s_S' % tag]).max() <= 1e-14


def test_oracle_matches_host_one_body(library):
    """The product's host S, T (napmo_basis_one_body) equal the oracle's."""
    import ints as I
    import oracle as O
    from napmo_b200 import cext
    from napmo_b200.system import build_system
    for atoms in (H2O, HCN):
        cs = [np.array(x) / BOHR for _, x in atoms]
        fb = O.flat_basis(cs, [s for s, _ in atoms], library, 'CC-PVDZ')
        S, T, _ = I.one_body(fb, [])
        b = build_system(atoms, 'CC-PVDZ')['e-']['basis']
        n = fb['nf']
        S2, T2 = np.zeros((n, n)), np.zeros((n, n))
        cext.checked(cext.lib.napmo_basis_one_body(b._this, S2, T2))
        assert np.abs(S - S2).max() <= 1e-13
        assert np.abs(T - T2).max() <= 1e-13 * np.abs(T).max()


def test_libint_interface_bookkeeping():
    """nAPMO's libint interface object: bases and point charges are
    collected on the host (no device work)."""
    from napmo_b200 import cext
    from napmo_b200.system import build_system
    ms = build_system(H2O, 'CC-PVDZ')
    lint = cext.lib.LibintInterface_new(0)
    assert lint
    cext.lib.LibintInterface_add_basis(lint, ms['e-']['basis']._this)
    for pc in ms.point_charges:
        cext.lib.LibintInterface_add_pointcharges(lint, pc['atomic_number'],
                                                 np.asarray(pc['origin'], np.float64))
    assert cext.lib.LibintInterface_get_nbasis(lint) == 25
    cext.lib.LibintInterface_del(lint)


def test_oracle_translation_invariance(library):
    """S and T of a molecule do not change when it moves; V does not change
    when the charges move with it."""
    import ints as I
    import oracle as O
    cs = [np.array(x) / BOHR for _, x in H2O]
    shift = np.array([0.7, -1.3, 2.1])
    out = []
    for c in (cs, [x + shift for x in cs]):
        fb = O.flat_basis(c, [s for s, _ in H2O], library, 'STO-3G')
        out.append(I.one_body(fb, [(Z, x) for Z, x in zip([8.0, 1.0, 1.0], c)]))
    for a, b in zip(*out):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
