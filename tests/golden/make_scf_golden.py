"""Converged grid SCFs of the oracle (oracle/scf.py) at the two SCF
configurations, written to tests/golden/scf_oracle.json (+ .npz densities):

  C1  RHF of H2O/cc-pVDZ (O at the origin, H at (0, +-0.757, 0.587) A),
      50 radial x 110 Lebedev per atom, grid J and orbital-pair exchange;
  C2  APMO-RHF of HCN (H at 0, C at 1.066 A, N at 2.222 A along z), electrons
      in cc-pVDZ, the H nucleus quantum in the even-tempered 5s5p basis
      (exponents 4..64), 100 radial x 302 Lebedev per atom;
  uhf_oh         UHF of the OH radical (O at 0, H at 0.97 A along z; doublet),
                 cc-pVDZ, 50 x 110;
  apmo_uhf_oh    APMO-UHF of the OH radical (doublet) with the H nucleus
                 quantum (5s5p), 50 x 110;
  uks_oh         unrestricted Kohn-Sham of the OH radical (doublet) with the
                 spin-polarised LDA (Slater + VWN5 of the two spin densities),
                 cc-pVDZ, 50 x 110.

Both stop at |dE| < 1e-9 Eh with max |X^T (FDS - SDF) X| < 1e-4 (the rule of
napmo_b200.scf), DIIS with 6 vectors.  The GPU tests compare the device
drivers' converged energies and iteration counts with these.  The C2 SCF
takes about ten minutes on 8 host cores.

Usage: python tests/golden/make_scf_golden.py [c1] [c2] [uhf_oh] [apmo_uhf_oh] [uks_oh]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
sys.path.insert(0, os.path.join(ROOT, 'tests'))

import scf as OS  # noqa: E402
from helpers import H2O, HCN  # noqa: E402

OH = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.0, 0.97))]

TOL = 1e-9


def load():
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'basis.json')) as f:
        lib = json.load(f)
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'elements.json')) as f:
        el = json.load(f)
    return lib, el


def run(case):
    lib, el = load()
    t0 = time.perf_counter()
    if case == 'c1':
        res = OS.GridRHF(H2O, lib, el, 50, 110).run(tol=TOL)
        arrays = {'c1_D': res['D']}
    elif case == 'uhf_oh':
        res = OS.GridMultiSCF(OH, lib, el, (), 50, 110).run(tol=TOL)
        arrays = {'uhf_oh_Da': res['D'][0], 'uhf_oh_Db': res['D'][1]}
    elif case == 'uks_oh':
        res = OS.GridMultiSCF(OH, lib, el, (), 50, 110, exchange='lda').run(tol=TOL)
        arrays = {}
    elif case == 'apmo_uhf_oh':
        res = OS.GridMultiSCF(OH, lib, el, (1,), 50, 110).run(tol=TOL)
        arrays = {}
    else:
        res = OS.GridAPMO(HCN, lib, el, (0,), 100, 302).run(tol=TOL)
        arrays = {'c2_De': res['De'], 'c2_Dn': res['Dn']}
    rec = dict(energy=res['energy'], iterations=res['iterations'],
               converged=res['converged'], tol=TOL, seconds=time.perf_counter() - t0,
               history=[list(h) for h in res['history']])
    return rec, arrays


def main(cases):
    jpath = os.path.join(HERE, 'scf_oracle.json')
    npath = os.path.join(HERE, 'scf_oracle.npz')
    out = json.load(open(jpath)) if os.path.exists(jpath) else {}
    arrs = dict(np.load(npath)) if os.path.exists(npath) else {}
    for c in cases:
        rec, a = run(c)
        out[c] = rec
        arrs.update(a)
        print('%s: E = %.12f Eh, %d iterations, %.1f s' % (c, rec['energy'], rec['iterations'],
                                                          rec['seconds']))
    with open(jpath, 'w') as f:
        json.dump(out, f, indent=1)
    np.savez_compressed(npath, **arrs)


if __name__ == '__main__':
    main([a for a in sys.argv[1:]] or ['c1', 'c2'])
