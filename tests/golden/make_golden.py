"""Generate the golden fixtures of tests/golden from the nAPMO tree.

* ``known_answers.json``: the numbers nAPMO's own tests assert, read from
  the test files themselves (file and the asserted value).
* ``reference_vectors.npz``: outputs of nAPMO's own compiled sources
  (oracle/_ref/libnapmo_ref.so, built by oracle/Makefile) on small seeded
  inputs: Lebedev rules, Chebyshev/Power radial transforms, Cartesian GTO
  values and overlap matrices (H2O/cc-pVDZ, HCN/cc-pVDZ), spline derivatives,
  FEM assembly and the multipole evaluation of a decomposition.

Usage: python tests/golden/make_golden.py [/path/to/nAPMO] [--answers-only]
"""
import json
import os
import re
import sys
from ctypes import c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def known_answers(ref):
    def grab(path, pattern, cast=float, flags=0):
        with open(os.path.join(ref, path)) as f:
            text = f.read()
        m = re.search(pattern, text, flags)
        if m is None:
            raise RuntimeError('pattern not found in %s' % path)
        return cast(m.group(1))

    def vec(path, name):
        with open(os.path.join(ref, path)) as f:
            text = f.read()
        m = re.search(name + r' = """(.*?)"""', text, re.S)
        return [float(x) for x in m.group(1).split()]

    out = {
        'coulomb_H_sto3g_100x110': {
            'value': grab('napmo/grids/test/test_coulomb.py', r'allclose\(integral, ([0-9.]+)\)'),
            'source': 'napmo/grids/test/test_coulomb.py'},
        'basis_H_sto3g_phi0': {
            'value': grab('napmo/gto/test/test_basis_set.py', r'np.array\(\[\[([0-9.]+)\]\]\)'),
            'source': 'napmo/gto/test/test_basis_set.py'},
        's_norm_zeta05': {
            'value': grab('napmo/gto/test/test_primitive_gaussian.py',
                          r'test.normalization, ([0-9.]+)\)'),
            'source': 'napmo/gto/test/test_primitive_gaussian.py'},
        'fz3_norm_zeta05': {
            'value': float(re.findall(r'test.normalization, ([0-9.]+)\)',
                                      open(os.path.join(ref, 'napmo/gto/test/test_primitive_gaussian.py')).read())[1]),
            'source': 'napmo/gto/test/test_primitive_gaussian.py'},
        'fz3_value_at_111': {
            'value': grab('napmo/gto/test/test_primitive_gaussian.py',
                          r'compute\(np.ones\(\[1, 3\]\)\), ([0-9.]+)\)'),
            'source': 'napmo/gto/test/test_primitive_gaussian.py'},
        'radial_He_50_points': {
            'value': vec('napmo/wavefunction/test/test_kinetic.py', 'rdat'),
            'source': 'napmo/wavefunction/test/test_kinetic.py'},
        'deriv2_He_50_input': {
            'value': vec('napmo/wavefunction/test/test_kinetic.py', 'test'),
            'source': 'napmo/wavefunction/test/test_kinetic.py'},
        'deriv2_He_50': {
            'value': vec('napmo/wavefunction/test/test_kinetic.py', 'gold'),
            'source': 'napmo/wavefunction/test/test_kinetic.py'},
        'becke_He_sto3g_300x110_energy': {
            'value': grab('napmo/wavefunction/test/test_psi_numeric_becke_He.py',
                          r'allclose\(E_tot, (-[0-9.]+), rtol=1e-5\)'),
            'rtol': 1e-5,
            'source': 'napmo/wavefunction/test/test_psi_numeric_becke_He.py'},
        'becke_He_sto3g_300x110_grid_energy': {
            'value': grab('napmo/wavefunction/test/test_psi_numeric_becke_He.py',
                          r'GRID: (-[0-9.]+) \(300x110\)'),
            'source': 'napmo/wavefunction/test/test_psi_numeric_becke_He.py (docstring: the '
                      'grid energy of this algorithm on 300x110)'},
        'becke_H2_sto3g_100x110_energy': {
            'value': grab('napmo/wavefunction/test/test_psi_numeric_becke_H2.py',
                          r'GRID: (-[0-9.]+) \(100x110\)'),
            'rtol': 1e-2,
            'source': 'napmo/wavefunction/test/test_psi_numeric_becke_H2.py'},
        'lebedev_110_order': {'value': 17, 'source': 'napmo/grids/test/test_lebedev.py'},
        'multigrid_common_points': {'value': 5500, 'source': 'napmo/grids/test/test_multi_grid.py'},
    }
    return out


def reference_vectors():
    import oracle as O
    r = O.ref_lib()
    if r is None:
        raise RuntimeError('oracle/_ref/libnapmo_ref.so missing: run make -C oracle')
    out = {}
    for order in (6, 14, 26, 38, 50, 74, 86, 110, 146, 170, 194, 230, 266, 302, 350, 434,
                  590, 770, 974, 1202, 1454, 1730, 2030, 2354, 2702, 3074, 3470, 3890, 4334,
                  4802, 5294, 5810):
        x, y, z, w = (np.zeros(order) for _ in range(4))
        r.ld_by_order(order, x, y, z, w)
        out['lebedev_%d' % order] = np.stack([x, y, z, w], axis=1)
    for name, radii, n in (('cheb_H_100', 0.5858151015155881, 100),
                           ('cheb_O_50', 1.2472192483880264, 50),
                           ('cheb_C_75', 1.4069648596390618, 75)):
        rt = r.ChebyshevRTransform_new(radii, n)
        t = np.arange(n, dtype=np.float64)
        out['rt_' + name] = np.array([[r.RTransform_radius(rt, x), r.RTransform_deriv(rt, x),
                                       r.RTransform_deriv2(rt, x), r.RTransform_deriv3(rt, x)]
                                      for x in t])
    rt = r.PowerRTransform_new(1e-3, 2e1, 100)
    out['rt_power_100'] = np.array([[r.RTransform_radius(rt, x), r.RTransform_deriv(rt, x)]
                                    for x in np.arange(100.0)])
    # GTO values through nAPMO's own BasisSet (Cartesian, file order)
    lib = json.load(open(os.path.join(ROOT, 'napmo_b200', 'data', 'basis.json')))
    rng = np.random.default_rng(20261203)
    for tag, atoms in (('h2o', [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 1.430522, 1.109257)),
                                ('H', (0.0, -1.430522, 1.109257))]),
                       ('hcn', [('H', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 2.014455)),
                                ('N', (0.0, 0.0, 4.199027))])):
        keep = []
        cont = []
        for sym, xyz in atoms:
            for (lval, exps, coefs) in lib['CC-PVDZ'][sym]:
                for k, i in enumerate(reversed(range(lval + 1))):
                    for j in range(k + 1):
                        prims = []
                        for e, c in zip(exps, coefs):
                            p = r.PrimitiveGaussian_new(np.array([i, k - j, j], np.int32),
                                                        np.array(xyz, np.float64), e, c)
                            prims.append(p)
                        keep.append(prims)
                        arr = np.array(prims, dtype=c_void_p)
                        keep.append(arr)
                        cont.append(r.ContractedGaussian_new(arr, len(prims)))
        carr = np.array(cont, dtype=c_void_p)
        bs = r.BasisSet_new(carr, len(cont))
        pts = np.ascontiguousarray(rng.normal(scale=1.5, size=(64, 3)))
        phi = np.zeros((64, len(cont)))
        r.BasisSet_compute(bs, pts, phi, 64)
        out['gto_%s_points' % tag] = pts
        out['gto_%s_phi' % tag] = phi
        # overlap matrix by nAPMO's own contracted overlap (gto.cpp, ints/overlap.cpp)
        out['ints_%s_S' % tag] = np.array([[r.ContractedGaussian_overlap(ci, cj) for cj in cont]
                                           for ci in cont])
    # spline derivatives and FEM assembly on a random case
    y = np.ascontiguousarray(rng.normal(size=40))
    dt = np.zeros(40)
    r.solve_cubic_spline_system(y, dt, 40)
    out['spline_y'], out['spline_dt'] = y, dt
    n = 12
    b, a, f = (np.ascontiguousarray(rng.normal(size=2 * n)) for _ in range(3))
    bcs = np.array([0.3, np.nan, -0.7, np.nan])
    coeffs = np.zeros((2 * n, 2 * n))
    rhs = np.zeros(2 * n)
    r.build_ode2(b, a, f, bcs, coeffs, rhs, n)
    out['ode_b'], out['ode_a'], out['ode_f'] = b, a, f
    out['ode_coeffs'], out['ode_rhs'] = coeffs, rhs
    # multipole evaluation of a random decomposition (lmax 4) on a Chebyshev grid
    lmax, nrad, radii = 4, 30, 1.2472192483880264
    rt = r.ChebyshevRTransform_new(radii, nrad)
    ys = np.ascontiguousarray(rng.normal(size=((lmax + 1) ** 2, nrad)))
    dts = np.ascontiguousarray(rng.normal(size=((lmax + 1) ** 2, nrad)))
    splines, keep2 = [], []
    c = 0
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            ext = r.PotentialExtrapolation_new(l)
            yy, dd = np.ascontiguousarray(ys[c]), np.ascontiguousarray(dts[c])
            keep2 += [yy, dd]
            splines.append(r.CubicSpline_new(yy, dd, ext, rt, nrad))
            c += 1
    sp = np.array(splines, dtype=c_void_p)
    center = np.array([0.1, -0.2, 0.3])
    pts = np.ascontiguousarray(rng.normal(scale=2.0, size=(200, 3)))
    pts[0] = center + np.array([1e-5, 0.0, 0.0])      # left extrapolation
    outv = np.zeros(200)
    cell = r.Cell_new(None, 0)
    r.eval_decomposition_grid(sp, center, outv, pts, cell, len(splines), 200)
    out['dec_y'], out['dec_dt'], out['dec_center'], out['dec_points'] = ys, dts, center, pts
    out['dec_radii'] = np.array([radii, nrad, lmax], dtype=np.float64)
    out['dec_out'] = outv
    return out


if __name__ == '__main__':
    args = [a for a in sys.argv[1:] if not a.startswith('--')]
    ref = args[0] if args else os.environ.get('NAPMO_REFERENCE')
    if not ref:
        sys.exit('usage: make_golden.py <nAPMO source tree> [--answers-only] '
                 '(or set NAPMO_REFERENCE)')
    with open(os.path.join(HERE, 'known_answers.json'), 'w') as f:
        json.dump(known_answers(ref), f, indent=1)
    if '--answers-only' not in sys.argv:
        np.savez_compressed(os.path.join(HERE, 'reference_vectors.npz'), **reference_vectors())
    print('wrote known_answers.json' +
          ('' if '--answers-only' in sys.argv else ' and reference_vectors.npz'))
