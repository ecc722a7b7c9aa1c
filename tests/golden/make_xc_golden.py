"""Subsample nAPMO's LDA fixtures into tests/golden/xc_lda.npz.

nAPMO's napmo/functional/test/ holds 22,000 densities (rho.txt) and the
LibXC outputs its Functional('Li') returned for them: lda_x and lda_c_vwn
energies per particle (x_zk.txt, c_zk.txt) and potentials (x_vrho.txt,
c_vrho.txt).  Kept: every 10th point, plus every point below 1e-10 (zeros,
denormal-range values and the cut of the smallest densities).

Usage: python tests/golden/make_xc_golden.py /path/to/nAPMO (or NAPMO_REFERENCE set)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    d = os.path.join(ref, 'napmo', 'functional', 'test')
    arrs = {k: np.fromfile(os.path.join(d, k + '.txt'), sep=' ')
            for k in ('rho', 'x_zk', 'x_vrho', 'c_zk', 'c_vrho')}
    rho = arrs['rho']
    keep = np.zeros(rho.size, bool)
    keep[::10] = True
    keep |= rho < 1e-10
    out = {k: v[keep] for k, v in arrs.items()}
    out['index'] = np.flatnonzero(keep)
    np.savez_compressed(os.path.join(HERE, 'xc_lda.npz'), **out)
    print('kept %d of %d points' % (keep.sum(), rho.size))


if __name__ == '__main__':
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('NAPMO_REFERENCE')
    if not ref:
        sys.exit('usage: make_xc_golden.py <nAPMO source tree> (or set NAPMO_REFERENCE)')
    main(ref)
