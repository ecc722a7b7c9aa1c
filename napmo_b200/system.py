"""Molecular systems: species dictionaries in nAPMO's layout and the
geometries of the workloads this package is measured on.

A species dict carries what the grid and SCF layers read
(napmo/system/molecular_system.py:32-214): ``symbol``, ``particles``
(centres with ``symbol`` and ``origin`` in bohr), ``basis`` (BasisSet over
all centres), ``size`` (number of particles), ``occupation``, ``eta``,
``kappa``, ``charge``.
"""
import math

import numpy as np

from .grids import ELEMENTS
from .gto import BasisSet

BOHR_TO_ANGSTROM = 0.52917724924   # napmo/data/constants.py

# species constants (napmo/data/elementary_particles.json,
# coupling_constants.json): eta, kappa, particles fraction, charge
ELECTRON = dict(eta=2.0, kappa=-1.0, particlesfraction=0.5, charge=-1.0)
NUCLEUS = dict(eta=1.0, kappa=-1.0, particlesfraction=1.0, charge=1.0)

# even-tempered 5s5p nuclear basis, exponents 4..64 bohr^-2 (ratio 2)
NUCLEAR_5S5P = [(0, [z], [1.0]) for z in (4.0, 8.0, 16.0, 32.0, 64.0)] + \
               [(1, [z], [1.0]) for z in (4.0, 8.0, 16.0, 32.0, 64.0)]


class MolecularSystem(dict):
    """Electrons on atoms (optionally some nuclei as quantum species)."""

    def __init__(self):
        super(MolecularSystem, self).__init__()
        self.point_charges = []
        self.charges = {}
        self.open_shell = False

    def set_charges(self, data, open_shell=False):
        """Charge and multiplicity per species (molecular_system.py:214-290):
        data = {'e-': {'charge': c, 'multiplicity': m}} adds c particles to
        the species (c = -1 removes an electron) and fixes its multiplicity
        (default 1 or 2 by parity).  The electrons are open shell when the
        alpha and beta counts differ or `open_shell` is set; the unrestricted
        drivers then treat them as e-alpha and e-beta."""
        e = self['e-']
        for key, val in data.items():
            if key not in self:
                raise ValueError('Impossible to set %s charges: particle does not exist' % key)
            self.charges[key] = dict(charge=int(val.get('charge', 0)),
                                     multiplicity=int(val.get('multiplicity', 0) or 0))
        c = self.charges.get('e-', {})
        nel = int(round(e['size'])) + c.get('charge', 0)
        m = c.get('multiplicity') or (nel % 2) + 1
        unpaired = m - 1
        if (nel - unpaired) % 2 != 0 or nel < unpaired:
            raise ValueError('Bad charge / multiplicity')
        self.open_shell = bool(unpaired) or bool(open_shell)
        return self

    def _species(self, symbol, consts):
        sp = self.setdefault(symbol, dict(symbol=symbol, particles=[], size=0, occupation=0,
                                          basis=None, **consts))
        return sp

    def add_atom(self, symbol, origin, units='ANGSTROMS', basis_name=None, quantum=False,
                 nuclear_shells=None):
        origin = np.array(origin, dtype=np.float64)
        if units.upper().startswith('ANGSTROM'):
            origin = origin / BOHR_TO_ANGSTROM
        Z = ELEMENTS[symbol]['atomic_number']
        e = self._species('e-', ELECTRON)
        e['particles'].append(dict(symbol=symbol, origin=origin, atomic_number=Z))
        if basis_name:
            b = BasisSet(basis_name, symbol, origin=origin)
            if e['basis'] is None:
                e['basis'] = BasisSet(basis_name, 'e-')
            e['basis'].update(b)
        e['size'] += Z
        e['occupation'] = int(e['size'] * e['particlesfraction'])
        if quantum:
            nsym = symbol + '_1'
            n = self._species(nsym, NUCLEUS)
            n['particles'].append(dict(symbol=nsym, origin=origin, atomic_number=Z))
            b = BasisSet('NUCLEAR-5S5P', nsym, origin=origin,
                         shells=nuclear_shells or NUCLEAR_5S5P)
            if n['basis'] is None:
                n['basis'] = BasisSet('NUCLEAR-5S5P', nsym)
            n['basis'].update(b)
            n['size'] += 1
            n['occupation'] = n['size']
        else:
            self.point_charges.append(dict(atomic_number=Z, origin=origin))
        return self

    def species(self, symbol='e-'):
        return self[symbol]


# ------------------------------------------------------------ geometries (A)
def h2o_geometry():
    return [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.757, 0.587)), ('H', (0.0, -0.757, 0.587))]


def hcn_geometry():
    return [('H', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 1.066)), ('N', (0.0, 0.0, 2.222))]


def alkane_geometry(ncarbon=20, cc=1.54, ch=1.09):
    """Linear (all-trans) alkane CnH2n+2 with tetrahedral angles."""
    theta = math.acos(-1.0 / 3.0)            # 109.47 deg
    half = theta / 2.0
    dz = cc * math.sin(half)                 # advance along the chain axis
    dy = cc * math.cos(half)                 # zig-zag amplitude
    carbons = []
    for i in range(ncarbon):
        carbons.append(np.array([0.0, (dy / 2.0) * (1 if i % 2 == 0 else -1), i * dz]))
    atoms = [('C', tuple(c)) for c in carbons]
    # two H per carbon in the plane perpendicular to the backbone plane,
    # plus one extra H on each chain end
    hx = ch * math.sin(half)
    for i, c in enumerate(carbons):
        side = 1.0 if i % 2 == 0 else -1.0
        hy = ch * math.cos(half) * side
        atoms.append(('H', (hx, c[1] + hy, c[2])))
        atoms.append(('H', (-hx, c[1] + hy, c[2])))
    # terminal H: where the zig-zag would put the next carbon (tetrahedral)
    for end, virt in ((0, -1), (ncarbon - 1, ncarbon)):
        c = carbons[end]
        nxt = np.array([0.0, (dy / 2.0) * (1 if virt % 2 == 0 else -1), virt * dz])
        d = (nxt - c) / np.linalg.norm(nxt - c)
        atoms.append(('H', tuple(c + ch * d)))
    return atoms


def build_system(atoms, basis='CC-PVDZ', quantum=()):
    ms = MolecularSystem()
    for i, (sym, xyz) in enumerate(atoms):
        ms.add_atom(sym, xyz, basis_name=basis, quantum=(i in quantum))
    return ms


def random_chain(rng, natom, symbols=('H', 'C', 'N', 'O')):
    """Random valence-respecting chain of ``natom`` atoms (bond 1.0-1.5 A,
    non-bonded distances >= 1.0 A), ends capped by H where possible."""
    valence = {'H': 1, 'C': 4, 'N': 3, 'O': 2}
    while True:
        syms = []
        for i in range(natom):
            if i == 0 or i == natom - 1:
                syms.append(symbols[rng.integers(len(symbols))])
            else:
                syms.append(symbols[1 + rng.integers(len(symbols) - 1)])  # no H inside
        if natom > 1 and (valence[syms[0]] < 1 or valence[syms[-1]] < 1):
            continue
        pos = [np.zeros(3)]
        ok = True
        for i in range(1, natom):
            for _try in range(200):
                v = rng.normal(size=3)
                v /= np.linalg.norm(v)
                p = pos[-1] + v * rng.uniform(1.0, 1.5)
                if all(np.linalg.norm(p - q) >= 1.0 for q in pos[:-1]):
                    pos.append(p)
                    break
            else:
                ok = False
                break
        if ok:
            return list(zip(syms, [tuple(p) for p in pos]))


ANGULAR_SIZES = (110, 146, 170, 194, 230, 266, 302, 350, 434, 590)


def random_batch(nmol=64, seed=20261203, natom=(3, 30), nrad=(50, 100), angular=ANGULAR_SIZES):
    """Seeded batch of random {H, C, N, O} chains (random_chain) with grid
    sizes drawn per atom: nrad uniform in [nrad[0], nrad[1]], nang from
    ``angular``.  Returns a list of {'atoms', 'nrad', 'nang'}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nmol):
        na = int(rng.integers(natom[0], natom[1] + 1))
        atoms = random_chain(rng, na)
        nr = [int(rng.integers(nrad[0], nrad[1] + 1)) for _ in atoms]
        ng = [int(angular[int(rng.integers(len(angular)))]) for _ in atoms]
        out.append({'atoms': atoms, 'nrad': nr, 'nang': ng})
    return out
