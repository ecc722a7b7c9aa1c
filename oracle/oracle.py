"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py use it as the checker; the napmo_b200 package
never imports it).

Python side of the CPU restatement of nAPMO's grid-quadrature path:
  * ctypes wrappers of oracle/liboracle.so (oracle.c, the C restatement);
  * ctypes wrappers of oracle/_ref/libnapmo_ref.so (nAPMO's own compilable
    sources, built by oracle/Makefile) where available;
  * the Poisson driver of napmo/grids/poisson_solver.py:18-118 and
    napmo/utilities/ode2.py:35-118 restated for NumPy 2 (np.nan instead of
    np.NaN), with scipy's sparse LU as in the reference;
  * the density of napmo/wavefunction/psi_hybrid.py:144-150 and the nuclear
    potential of napmo/wavefunction/nnuclear.py:15-37.
"""
import ctypes
import os
from ctypes import c_bool, c_double, c_int, c_long, c_void_p

import numpy as np
import numpy.ctypeslib as npct

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, 'liboracle.so')
REF_SO = os.path.join(HERE, '_ref', 'libnapmo_ref.so')

a1d = npct.ndpointer(dtype=np.float64, ndim=1, flags='C_CONTIGUOUS')
a2d = npct.ndpointer(dtype=np.float64, ndim=2, flags='C_CONTIGUOUS')
a1i = npct.ndpointer(dtype=np.int32, ndim=1, flags='C_CONTIGUOUS')
a1l = npct.ndpointer(dtype=np.int64, ndim=1, flags='C_CONTIGUOUS')
aptr = npct.ndpointer(c_void_p, flags='C_CONTIGUOUS')

BOHR_TO_ANGSTROM = 0.52917724924


def build():
    """Compile liboracle.so (and _ref when the reference tree is present)."""
    import subprocess
    subprocess.check_call(['make', '-s', '-C', HERE])


def _load_oracle():
    if not os.path.exists(ORACLE_SO):
        build()
    lib = ctypes.CDLL(ORACLE_SO)
    sig = {
        'orc_radial_grid': (None, [c_int, c_double, c_double, c_int, a1d, a1d]),
        'orc_cheb_radius': (c_double, [c_double, c_int, c_double]),
        'orc_cheb_deriv': (c_double, [c_double, c_int, c_double]),
        'orc_cheb_deriv2': (c_double, [c_double, c_int, c_double]),
        'orc_cheb_deriv3': (c_double, [c_double, c_int, c_double]),
        'orc_cheb_inv': (c_double, [c_double, c_int, c_double]),
        'orc_lebedev': (c_int, [c_int, a1d, a1d, a1d, a1d]),
        'orc_atomic_grid': (None, [c_int, a1d, a1d, c_int, a1d, a1d, a1d, a1d, a1d, a2d, a1d]),
        'orc_becke_weights': (None, [c_int, c_int, a1d, a2d, a2d, a1i, a1d]),
        'orc_prim_norm': (c_double, [a1i, c_double]),
        'orc_basis_compute': (None, [c_int, a1i, a1d, a1i, a1i, a1d, a1d, c_int, a2d, a2d]),
        'orc_density': (None, [c_int, c_int, a2d, a2d, a1d]),
        'orc_quadrature': (None, [c_int, c_int, a2d, a1d, a1d, a1d, a2d]),
        'orc_spherical_expansion': (None, [c_int, c_int, a2d, a1d, a1d, a1d, c_int, a2d]),
        'orc_spline_dt': (None, [a1d, a1d, c_int]),
        'orc_spline_dt_many': (None, [a2d, a2d, c_int, c_int]),
        'orc_spherical_expansion_many': (None, [c_int, c_int, a2d, a1d, a1d, c_int, a2d, c_long,
                                                c_int, a2d]),
        'orc_build_ode2': (None, [a1d, a1d, a1d, a1d, a2d, a1d, c_long]),
        'orc_eval_decomposition': (None, [c_int, c_double, c_double, c_int, c_int, a2d, a2d,
                                          a1d, c_int, a2d, a1d]),
        'orc_eval_decomposition_many': (None, [c_int, c_double, c_double, c_int, c_int, c_int,
                                               a2d, a2d, a1d, c_int, a2d, a2d, c_long]),
        'orc_num_threads': (c_int, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


lib = _load_oracle()


def threads():
    return lib.orc_num_threads()


# ---------------------------------------------------------------- reference
def ref_lib():
    """nAPMO's own compiled sources, or None when oracle/_ref is absent."""
    if not os.path.exists(REF_SO):
        return None
    r = ctypes.CDLL(REF_SO)
    sig = {
        'ChebyshevRTransform_new': (c_void_p, [c_double, c_int]),
        'PowerRTransform_new': (c_void_p, [c_double, c_double, c_int]),
        'RTransform_radius': (c_double, [c_void_p, c_double]),
        'RTransform_deriv': (c_double, [c_void_p, c_double]),
        'RTransform_deriv2': (c_double, [c_void_p, c_double]),
        'RTransform_deriv3': (c_double, [c_void_p, c_double]),
        'RTransform_inv': (c_double, [c_void_p, c_double]),
        'ld_by_order': (None, [c_int, a1d, a1d, a1d, a1d]),
        'PrimitiveGaussian_new': (c_void_p, [a1i, a1d, c_double, c_double]),
        'PrimitiveGaussian_get_norma': (c_double, [c_void_p]),
        'ContractedGaussian_new': (c_void_p, [aptr, c_int]),
        'ContractedGaussian_get_norma': (c_double, [c_void_p]),
        'ContractedGaussian_overlap': (c_double, [c_void_p, c_void_p]),
        'BasisSet_new': (c_void_p, [aptr, c_int]),
        'BasisSet_compute': (None, [c_void_p, a2d, a2d, c_int]),
        'solve_cubic_spline_system': (None, [a1d, a1d, c_int]),
        'build_ode2': (None, [a1d, a1d, a1d, a1d, a2d, a1d, c_long]),
        'hermite_overlap2': (c_double, [c_long, c_long, c_bool, c_long, c_bool]),
        'hermite_overlap3': (c_double, [c_long, c_long, c_bool, c_long, c_bool, c_long, c_bool]),
        'dot_multi_moments': (None, [c_long, c_long, a1d, a2d, a1d, c_long, c_long, a1l, a2d,
                                     c_long]),
        'CubicSpline_new': (c_void_p, [a1d, a1d, c_void_p, c_void_p, c_int]),
        'CubicSpline_eval': (None, [c_void_p, a1d, a1d, c_int]),
        'PotentialExtrapolation_new': (c_void_p, [c_int]),
        'Cell_new': (c_void_p, [c_void_p, c_int]),
        'eval_decomposition_grid': (None, [aptr, a1d, a1d, a2d, c_void_p, c_long, c_long]),
        'fill_pure_polynomials': (c_long, [a1d, c_long]),
    }
    # functions declared without extern "C" in nAPMO carry C++ linkage
    mangled = {'ld_by_order': '_Z11ld_by_orderiPdS_S_S_',
               'hermite_overlap2': '_Z16hermite_overlap2llblb',
               'hermite_overlap3': '_Z16hermite_overlap3llblblb',
               'fill_pure_polynomials': '_Z21fill_pure_polynomialsPdl'}
    for name, (res, args) in sig.items():
        f = getattr(r, mangled.get(name, name))
        f.restype, f.argtypes = res, args
        setattr(r, name, f)
    return r


# --------------------------------------------------------------------- grids
def radial_grid(n, radii=None, power=None):
    """Chebyshev (radii) or Power ((rmin, rmax)) radial points and weights."""
    r, w = np.zeros(n), np.zeros(n)
    if power is None:
        lib.orc_radial_grid(0, radii, 0.0, n, r, w)
    else:
        lib.orc_radial_grid(1, power[0], power[1], n, r, w)
    return r, w


def radial_derivs(n, radii):
    t = np.arange(n, dtype=np.float64)
    j1 = np.array([lib.orc_cheb_deriv(radii, n, x) for x in t])
    j2 = np.array([lib.orc_cheb_deriv2(radii, n, x) for x in t])
    j3 = np.array([lib.orc_cheb_deriv3(radii, n, x) for x in t])
    return j1, j2, j3


def lebedev(order):
    x, y, z, w = (np.zeros(order) for _ in range(4))
    n = lib.orc_lebedev(order, x, y, z, w)
    assert n == order, 'unknown Lebedev order %d' % order
    return np.stack([x, y, z], axis=1), w


class Atom(object):
    """One atomic grid of the oracle (radial-major points)."""

    def __init__(self, center, radii, nrad, nang):
        self.center = np.asarray(center, dtype=np.float64)
        self.radii, self.nrad, self.nang = radii, nrad, nang
        self.r, self.wr = radial_grid(nrad, radii)
        ang, aw = lebedev(nang)
        self.size = nrad * nang
        self.points = np.zeros((self.size, 3))
        self.weights = np.zeros(self.size)
        lib.orc_atomic_grid(nrad, self.r, self.wr, nang, np.ascontiguousarray(ang[:, 0]),
                            np.ascontiguousarray(ang[:, 1]), np.ascontiguousarray(ang[:, 2]),
                            aw, self.center, self.points, self.weights)


class Grid(object):
    """Molecular grid: concatenated atoms plus Becke weights (becke.cpp:12-176)."""

    def __init__(self, centers, radii, nrad, nang, becke=True):
        nc = len(centers)
        nr = nrad if isinstance(nrad, (list, tuple)) else [nrad] * nc
        na = nang if isinstance(nang, (list, tuple)) else [nang] * nc
        self.atoms = [Atom(centers[i], radii[i], nr[i], na[i]) for i in range(nc)]
        self.origin = np.ascontiguousarray(np.array(centers, dtype=np.float64).reshape(nc, 3))
        self.radii = np.array(radii, dtype=np.float64)
        self.points = np.ascontiguousarray(np.concatenate([a.points for a in self.atoms]))
        self.weights = np.ascontiguousarray(np.concatenate([a.weights for a in self.atoms]))
        self.size = self.points.shape[0]
        self.offsets = np.cumsum([0] + [a.size for a in self.atoms]).astype(np.int32)
        self.becke = np.zeros(self.size)
        if becke:
            lib.orc_becke_weights(nc, self.size, self.radii, self.origin, self.points,
                                  self.offsets, self.becke)

    def becke_sample(self, index):
        """Becke weights of the grid points `index` only (the per-point
        computation of becke.cpp:128-171 with each point's owning atom)."""
        index = np.asarray(index, dtype=np.int64)
        owner = np.searchsorted(self.offsets, index, side='right') - 1
        order = np.argsort(owner, kind='stable')
        pts = np.ascontiguousarray(self.points[index[order]])
        counts = np.bincount(owner, minlength=len(self.atoms))
        offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        out = np.zeros(len(index))
        lib.orc_becke_weights(len(self.atoms), len(index), self.radii, self.origin, pts, offs, out)
        res = np.empty(len(index))
        res[order] = out
        return res

    def integrate(self, f):
        return float(np.sum(f * self.becke * self.weights))


# ---------------------------------------------------------------------- basis
def flat_basis(centers, symbols, library, basis_name):
    """Flat description of the Cartesian basis over all centres, in nAPMO's
    function order (napmo/gto/basis_set.py:122-143)."""
    ls, origins, nprim, off, zeta, coeff = [], [], [], [], [], []
    for c, sym in zip(centers, symbols):
        shells = library[basis_name][sym]
        for (lval, exps, coefs) in shells:
            for k, i in enumerate(reversed(range(lval + 1))):
                for j in range(k + 1):
                    ls += [i, k - j, j]
                    origins += list(c)
                    off.append(len(zeta))
                    nprim.append(len(exps))
                    zeta += list(exps)
                    coeff += list(coefs)
    return dict(l=np.array(ls, np.int32), origin=np.array(origins, np.float64),
                nprim=np.array(nprim, np.int32), off=np.array(off, np.int32),
                zeta=np.array(zeta, np.float64), coeff=np.array(coeff, np.float64),
                nf=len(nprim))


def basis_compute(fb, points):
    """phi [npoint][nf] (BasisSet_compute layout)."""
    points = np.ascontiguousarray(points, dtype=np.float64)
    out = np.zeros((points.shape[0], fb['nf']))
    lib.orc_basis_compute(fb['nf'], fb['l'], fb['origin'], fb['nprim'], fb['off'], fb['zeta'],
                          fb['coeff'], points.shape[0], points, out)
    return out


def density(phi_t, D):
    """rho from phi [n][N] and D [n][n]."""
    n, N = phi_t.shape
    rho = np.zeros(N)
    lib.orc_density(n, N, np.ascontiguousarray(phi_t), np.ascontiguousarray(D), rho)
    return rho


def quadrature(phi_t, C, becke, weights):
    """F_ij = sum_p phi_i phi_j C becke w (nwavefunction_compute_coupling)."""
    n, N = phi_t.shape
    F = np.zeros((n, n))
    lib.orc_quadrature(n, N, np.ascontiguousarray(phi_t), np.ascontiguousarray(C, np.float64),
                       np.ascontiguousarray(becke), np.ascontiguousarray(weights), F)
    return F


def nuclear_potential(points, charges):
    """sum_A Z_A / |r - R_A| (nnuclear.py:15-37)."""
    v = np.zeros(points.shape[0])
    for (Z, R) in charges:
        v += Z / np.sqrt(((np.asarray(R) - points) ** 2).sum(axis=1))
    return v


# -------------------------------------------------------------------- Poisson
def spherical_expansion(atom, f, lmax):
    lsize = (lmax + 1) ** 2
    out = np.zeros((atom.nrad, lsize))
    lib.orc_spherical_expansion(atom.nrad, atom.nang, atom.points, atom.weights, atom.center,
                                np.ascontiguousarray(f, dtype=np.float64), lmax, out)
    return out


def _spline_dt(y):
    dt = np.zeros_like(y)
    lib.orc_spline_dt(np.ascontiguousarray(y), dt, y.shape[0])
    return dt


def poisson_solver(grid, dens, lmax):
    """U[atom] = (y [lsize][nrad], dt [lsize][nrad]) of the potential splines
    (poisson_solver.py:18-118 with solve_ode2 of ode2.py:35-118)."""
    from scipy.sparse import csc_matrix
    from scipy.sparse.linalg import spsolve
    dens = dens * grid.becke
    PI_4 = 4.0 * np.pi
    U = []
    off = 0
    for atom in grid.atoms:
        p = dens[off:off + atom.size].copy()
        sph = spherical_expansion(atom, p, lmax)
        radii = atom.r
        n = atom.nrad
        j1, j2, j3 = radial_derivs(n, atom.radii)
        radii2 = radii * radii
        radii3 = radii2 * radii
        b_y, b_dx = 2 / radii, -2 / radii2
        ys, dts = [], []
        for l in range(lmax + 1):
            radiiL = radii ** l
            radiiLm1 = radii ** (-l - 1)
            l2l = l * (l + 1)
            radiiVmax = 1.0 / radii[-1] ** (l + 1) / (2 * l + 1)
            radiiVmin = radii[0] ** l / (2 * l + 1)
            a_y, a_dx = -l2l / radii2, 2 * l2l / radii3
            for m in range(-l, l + 1):
                aux = np.ascontiguousarray(sph[:, l * l + m + l])
                rho_dt = _spline_dt(aux)
                rho_dx = rho_dt / j1
                fy = -PI_4 * aux
                fd = -PI_4 * rho_dx
                V_rmax = float(np.sum(aux * radiiL * atom.wr)) * radiiVmax
                V_rmin = float(np.sum(aux * radiiLm1 * atom.wr)) * radiiVmin
                # solve_ode2
                j1sq = j1 * j1
                by_new = j1 * b_y - j2 / j1
                bd_new = j2 * b_y + j1sq * b_dx + (j2 * j2 - j1 * j3) / j1sq
                ay_new = a_y * j1sq
                ad_new = (a_dx * j1sq + 2 * a_y * j2) * j1
                fy_new = fy * j1sq
                fd_new = (fd * j1sq + 2 * fy * j2) * j1
                merge = lambda u, v: np.ascontiguousarray(np.array([u, v]).T.ravel())
                bcs = np.array([V_rmin, np.nan, V_rmax, np.nan])
                coeffs = np.zeros((2 * n, 2 * n))
                rhs = np.zeros(2 * n)
                lib.orc_build_ode2(merge(by_new, bd_new), merge(ay_new, ad_new),
                                   merge(fy_new, fd_new), bcs, coeffs, rhs, n)
                sol = spsolve(csc_matrix(coeffs), rhs)
                ys.append(sol[::2].copy())
                dts.append((sol[1::2] / j1) * j1)
        U.append((np.array(ys), np.array(dts)))
        off += atom.size
    return U


def evaluate_decomposition(grid, atom_index, U_atom, out):
    atom = grid.atoms[atom_index]
    y, dt = U_atom
    lib.orc_eval_decomposition(0, atom.radii, 0.0, atom.nrad, y.shape[0],
                               np.ascontiguousarray(y), np.ascontiguousarray(dt), atom.center,
                               grid.size, grid.points, out)


def compute_coulomb(grid, dens, lmax):
    """V_H[dens] at every grid point (ntwobody.py:15-46)."""
    U = poisson_solver(grid, dens, lmax)
    J = np.zeros(grid.size)
    for i in range(len(grid.atoms)):
        evaluate_decomposition(grid, i, U[i], J)
    return J
