"""Grid side of the nAPMO-compatible Python API (``napmo.grids``).

Same class names, constructor arguments and properties as nAPMO's
``napmo/grids/*.py``; the objects live in libnapmo.so and every per-point
evaluation (Becke weights, spherical projections, the Poisson solve, the
multipole evaluation of potentials, grid integrals) runs on the GPU.
"""
import json
import os
from ctypes import byref, c_int, c_void_p

import numpy as np

from . import cext
from .cext import check, checked, NapmoError

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data')
with open(os.path.join(_DATA, 'elements.json')) as _f:
    ELEMENTS = json.load(_f)

_LEBEDEV_ORDER = {
    6: 3, 14: 5, 26: 7, 38: 9, 50: 11, 74: 13, 86: 15, 110: 17, 146: 19, 170: 21,
    194: 23, 230: 25, 266: 27, 302: 29, 350: 31, 434: 35, 590: 41, 770: 47, 974: 53,
    1202: 59, 1454: 65, 1730: 71, 2030: 77, 2354: 83, 2702: 89, 3074: 95, 3470: 101,
    3890: 107, 4334: 113, 4802: 119, 5294: 125, 5810: 131}


def lebedev_get_order(n):
    """Order of the Lebedev quadrature with ``n`` points (napmo/grids/lebedev.py:14-31)."""
    return _LEBEDEV_ORDER[n]


def _lib():
    return cext.lib


# ----------------------------------------------------------------- transforms
class RadialTransform(object):
    """r = f(t) on the uniform t-axis 0..size-1 (napmo/grids/radial_transform.py)."""

    def __init__(self):
        if not self._this:
            check()
            raise NapmoError('radial transform construction failed')
        self._size = _lib().RTransform_get_npoint(self._this)
        self._points = np.arange(self.size, dtype=np.float64)

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().RTransform_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def _apply(self, fn_scalar, fn_array, t):
        if isinstance(t, np.ndarray):
            t = np.ascontiguousarray(t, dtype=np.float64)
            out = np.zeros(t.shape[0], dtype=np.float64)
            fn_array(self._this, t, out, t.shape[0])
            return out
        return fn_scalar(self._this, float(t))

    def radius(self, t):
        return self._apply(_lib().RTransform_radius, _lib().RTransform_radius_array, t)

    def deriv(self, t):
        return self._apply(_lib().RTransform_deriv, _lib().RTransform_deriv_array, t)

    def deriv2(self, t):
        return self._apply(_lib().RTransform_deriv2, _lib().RTransform_deriv2_array, t)

    def deriv3(self, t):
        return self._apply(_lib().RTransform_deriv3, _lib().RTransform_deriv3_array, t)

    def inv(self, r):
        return self._apply(_lib().RTransform_inv, _lib().RTransform_inv_array, r)

    def radius_all(self, points=None):
        return self.radius(self._points if points is None else points)

    def deriv_all(self, points=None):
        return self.deriv(self._points if points is None else points)

    def deriv2_all(self, points=None):
        return self.deriv2(self._points if points is None else points)

    def deriv3_all(self, points=None):
        return self.deriv3(self._points if points is None else points)

    def inv_all(self, points):
        return self.inv(points)

    @property
    def size(self):
        return self._size


class IndentityRadialTransform(RadialTransform):
    def __init__(self, size):
        self._this = _lib().IdentityRTransform_new(size)
        super(IndentityRadialTransform, self).__init__()

    def to_string(self):
        return ' '.join(['IdentityRTransform', repr(self.size)])


class PowerRadialTransform(RadialTransform):
    """r_i = rmin (i + 1)^power with power = ln(rmax/rmin) / ln(size)."""

    def __init__(self, rmin, rmax, size):
        self._this = _lib().PowerRTransform_new(rmin, rmax, size)
        super(PowerRadialTransform, self).__init__()
        self._rmin = _lib().PowerRTransform_get_rmin(self._this)
        self._rmax = _lib().PowerRTransform_get_rmax(self._this)
        self._power = _lib().PowerRTransform_get_power(self._this)

    def to_string(self):
        return ' '.join(['PowerRTransform', repr(self.rmin), repr(self.rmax), repr(self.size)])

    rmin = property(lambda self: self._rmin)
    rmax = property(lambda self: self._rmax)
    power = property(lambda self: self._power)
    radii = property(lambda self: self._rmax)


class ChebyshevRadialTransform(RadialTransform):
    """Becke's r = radii (1 + x) / (1 - x), x = cos(pi i / (size + 1))."""

    def __init__(self, radii, size):
        self._this = _lib().ChebyshevRTransform_new(radii, size)
        super(ChebyshevRadialTransform, self).__init__()
        self._radii = _lib().ChebyshevRTransform_get_radii(self._this)

    def to_string(self):
        return ' '.join(['ChebyshevRTransform', repr(self.radii), repr(self.size)])

    radii = property(lambda self: self._radii)


def atomic_radius(symbol):
    """Radius nAPMO picks for the Chebyshev grid of ``symbol`` (radial.py:24-39)."""
    radii = ELEMENTS.get('H', {}).get('atomic_radii_2', 1.0)
    aux = symbol.find('_')
    if aux > 0:
        radii = ELEMENTS.get(symbol[0:aux], {}).get('atomic_radii', 1.0)
    if symbol in ELEMENTS:
        radii = ELEMENTS[symbol].get('atomic_radii', 1.0)
    return radii


# ---------------------------------------------------------------------- grids
class RadialGrid(object):
    def __init__(self, size=2, atomic_symbol='--', rtransform=None):
        self._symbol = atomic_symbol
        radii = atomic_radius(atomic_symbol)
        self._rtransform = rtransform
        if rtransform is None:
            self._rtransform = ChebyshevRadialTransform(radii, size)
        self._this = _lib().RadialGrid_new(self._rtransform._this, self._rtransform.radii)
        if not self._this:
            check()

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().RadialGrid_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def integrate(self, f, segments):
        f = np.ascontiguousarray(f, dtype=np.float64)
        return _lib().RadialGrid_integrate(self._this, segments, f)

    def deriv2(self, f):
        """(1/r) d2/dr2 (r f) by finite differences in the Chebyshev angle
        (radial.py, src/grid/radial.cpp:51-192)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.shape[0] != self.size:
            raise NapmoError('f must hold one value per radial point')
        ptr = _lib().RadialGrid_deriv2(self._this, f)
        if not ptr:
            check()
        out = cext.as_array(ptr, (self.size,)).copy()
        _lib().napmo_free_array(ptr)
        return out

    size = property(lambda self: _lib().RadialGrid_get_size(self._this))
    symbol = property(lambda self: self._symbol)
    radii = property(lambda self: _lib().RadialGrid_get_radii(self._this))
    rtransform = property(lambda self: self._rtransform)

    @property
    def points(self):
        return cext.as_array(_lib().RadialGrid_get_points(self._this), (self.size,))

    @property
    def weights(self):
        return cext.as_array(_lib().RadialGrid_get_weights(self._this), (self.size,))

    def zeros(self):
        return np.zeros(self.size)


class AngularGrid(object):
    """Lebedev-Laikov angular quadrature (unit vectors, weights sum to one)."""

    def __init__(self, lorder, spherical=False):
        self._this = _lib().AngularGrid_new(lorder)
        if not self._this:
            check()
        self._spherical = spherical
        if spherical:
            _lib().AngularGrid_spherical(self._this)

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().AngularGrid_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def integrate(self, *args):
        f = np.ascontiguousarray(np.concatenate(args), dtype=np.float64)
        return _lib().AngularGrid_integrate(self._this, len(args), f, None)

    lorder = property(lambda self: _lib().AngularGrid_get_lorder(self._this))
    spherical = property(lambda self: self._spherical)

    @property
    def points(self):
        return cext.as_array(_lib().AngularGrid_get_points(self._this), (self.lorder, 3))

    @property
    def weights(self):
        return cext.as_array(_lib().AngularGrid_get_weights(self._this), (self.lorder,))


class AtomicGrid(object):
    """Per-atom grid: points u_j r_i + R, weights w_ang,j w_rad,i, index i*nang + j."""

    def __init__(self, nrad, nang, origin, atomic_symbol, rtransform=None):
        self.radial_grid = RadialGrid(nrad, atomic_symbol, rtransform=rtransform)
        self.angular_grid = AngularGrid(nang)
        self._symbol = atomic_symbol
        origin = np.ascontiguousarray(origin, dtype=np.float64)
        self._this = _lib().AtomicGrid_new(self.angular_grid._this, self.radial_grid._this, origin)
        if not self._this:
            check()

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().AtomicGrid_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def spherical_expansion(self, lmax, f):
        """f_lm(r_i) = sqrt(4 pi (2l+1)) sum_j f w S_lm(u_j) / sum_j w, shape (nrad, lsize)."""
        if lmax < 0:
            raise ValueError('lmax can not be negative.')
        lsize = (lmax + 1) * (lmax + 1)
        f = np.ascontiguousarray(f, dtype=np.float64)
        ptr = _lib().AtomicGrid_spherical_expansion(self._this, f, lmax)
        check()
        out = cext.as_array(ptr, (self.radial_grid.size, lsize)).copy()
        _lib().napmo_free_array(ptr)
        return out

    def integrate(self, *args, **kwargs):
        segmented = kwargs.pop('segmented', False)
        args += (self.weights,)
        nfunc = len(args)
        if segmented:
            nseg, sseg = self.radial_grid.size, self.angular_grid.lorder
        else:
            nseg, sseg = 1, self.size
        f = np.ascontiguousarray(np.concatenate(args), dtype=np.float64)
        ptr = _lib().AtomicGrid_integrate(self._this, nfunc, nseg, sseg, f)
        out = cext.as_array(ptr, (nseg,)).copy()
        _lib().napmo_free_array(ptr)
        return out

    def spherical_average(self, *args):
        f = np.concatenate(args)
        s = self.integrate(segmented=True)
        output = self.integrate(f, segmented=True)
        output /= s
        return output

    @property
    def points(self):
        return cext.as_array(_lib().AtomicGrid_get_points(self._this), (self.size, 3))

    @property
    def weights(self):
        return cext.as_array(_lib().AtomicGrid_get_weights(self._this), (self.size,))

    @property
    def origin(self):
        return cext.as_array(_lib().AtomicGrid_get_origin(self._this), (3,))

    size = property(lambda self: _lib().AtomicGrid_get_size(self._this))
    radii = property(lambda self: _lib().AtomicGrid_get_radii(self._this))
    symbol = property(lambda self: self._symbol)


class Cell(object):
    """Non-periodic cell (the only kind molecular grids use)."""

    def __init__(self, rvecs=None):
        nvec = 0 if rvecs is None else len(rvecs)
        self._this = _lib().Cell_new(None, nvec)
        if not self._this:
            check()

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().Cell_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None


class BeckeGrid(object):
    """Molecular grid with Becke partition weights (napmo/grids/becke.py:19-164).

    ``species`` is a dict with ``particles`` = [{'origin': xyz (bohr),
    'symbol': str}, ...] and ``symbol``.  ``n_radial`` / ``n_angular`` may
    also be per-centre lists (atomic grids of different sizes).
    """

    def __init__(self, species, n_radial=40, n_angular=110, rtransform=None, file=None,
                 ablmax=None, abldep=None):
        assert isinstance(species, dict)
        centers = species.get('particles')
        ncenter = len(centers)
        self._symbol = species.get('symbol')
        if file is not None:
            from scipy.io import FortranFile
            f = FortranFile(file, 'r')
            size = f.read_ints(dtype=np.int64)[0]
            pw = f.read_reals(dtype=np.float64).reshape(int(size / 4), 4, order='F')
            pw = np.asanyarray(pw, order='C')
            self.atgrids = []
            self._this = _lib().BeckeGrid_from_points(pw, pw.shape[0], ncenter)
        else:
            ablmax = 0 if ablmax is None else ablmax
            abldep = 1.0e-6 if abldep is None else abldep
            self._nrad = n_radial
            self._nang = n_angular
            nr = n_radial if isinstance(n_radial, (list, tuple)) else [n_radial] * ncenter
            na = n_angular if isinstance(n_angular, (list, tuple)) else [n_angular] * ncenter
            self.atgrids = [AtomicGrid(nr[i], na[i], c.get('origin'), c.get('symbol'),
                                       rtransform=rtransform)
                            for i, c in enumerate(centers)]
            ptrs = np.array([a._this for a in self.atgrids], dtype=c_void_p)
            self._this = _lib().BeckeGrid_new(ptrs, ncenter, ablmax, abldep)
        if not self._this:
            check()
            raise NapmoError('BeckeGrid construction failed')

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().BeckeGrid_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def evaluate_decomposition(self, atom, cubic_splines, output, cell=None):
        """output += sum_lm spline_lm(|r - R|) Y_lm for one atom, at every grid point (GPU)."""
        if cell is None:
            cell = Cell(None)
        splines = np.array([cs._this for cs in cubic_splines], dtype=c_void_p)
        origin = np.ascontiguousarray(self.origin[atom, :])
        pts = np.ascontiguousarray(self.points)
        _lib().eval_decomposition_grid(splines, origin, output, pts, cell._this,
                                       len(cubic_splines), self.size)
        check()

    def integrate(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = _lib().BeckeGrid_integrate(self._this, f)
        return check(out)

    def set_centers(self, origins):
        """Moves the atomic grids to new centres (ncenter x 3, bohr) in place:
        points rebuilt around each centre, Becke weights recomputed, device
        buffers reused.  Plans on this grid need FockBuilder.refresh()."""
        origins = np.ascontiguousarray(np.asarray(origins, dtype=np.float64).reshape(-1, 3))
        checked(_lib().napmo_grid_set_centers(self._this, origins))

    def device_arrays(self):
        """Raw device pointers (x, y, z, w, becke weights) of the grid mirror."""
        ptrs = [c_void_p() for _ in range(5)]
        _lib().napmo_grid_device_arrays(self._this, *[byref(p) for p in ptrs])
        return [p.value for p in ptrs]

    def set_poisson_tolerance(self, tol):
        """Truncation tolerance (a.u.) of the potential evaluation of this
        grid's Poisson solves: 0 (default) sums every (l, m) <= lmax as nAPMO
        does; tol > 0 drops, per atom and radial interval, the highest
        l-blocks whose bounded contribution to any point stays <= tol."""
        cext.checked(_lib().napmo_grid_set_poisson_tolerance(self._this, float(tol)))

    def show(self):
        print('\nGrid Information:', self._symbol)
        print('-' * (18 + len(self._symbol)))
        print('Centers: ', self.ncenter)
        print('Size: ', self.size)

    @property
    def becke_weights(self):
        return cext.as_array(_lib().BeckeGrid_get_becke_weights(self._this), (self.size,))

    @property
    def points(self):
        return cext.as_array(_lib().BeckeGrid_get_points(self._this), (self.size, 3))

    @property
    def weights(self):
        return cext.as_array(_lib().BeckeGrid_get_weights(self._this), (self.size,))

    @property
    def origin(self):
        return cext.as_array(_lib().BeckeGrid_get_origin(self._this), (self.ncenter, 3))

    @property
    def radii(self):
        return cext.as_array(_lib().BeckeGrid_get_radii(self._this), (self.ncenter,))

    size = property(lambda self: _lib().BeckeGrid_get_size(self._this))
    ncenter = property(lambda self: _lib().BeckeGrid_get_ncenter(self._this))
    nrad = property(lambda self: self._nrad)
    nang = property(lambda self: self._nang)
    symbol = property(lambda self: self._symbol)


class MultiGrid(object):
    """Grids of several species and their bit-identical common points."""

    def __init__(self, nspecies):
        self._this = _lib().MultiGrid_new(nspecies)
        self._grids = []
        self._ids = {}

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().MultiGrid_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def add_grid(self, grid):
        gid = _lib().MultiGrid_add_grid(self._this, grid._this)
        self._grids.append(grid)
        self._ids[grid.symbol] = gid
        return gid

    def get_grid(self, symbol=None, gid=None):
        if gid is not None:
            return self._grids[gid] if gid < len(self._grids) else None
        i = self._ids.get(symbol)
        return None if i is None else self._grids[i]

    def get_grid_id(self, symbol):
        return self._ids.get(symbol)

    def get_common_points(self, sa, sb):
        a, b = self.get_grid_id(sa), self.get_grid_id(sb)
        if a is None or b is None:
            return None
        ptr = _lib().MultiGrid_get_common_index(self._this, a, b)
        check()
        n = _lib().MultiGrid_get_common_index_size(self._this, a, b)
        if n <= 0:
            return np.zeros((0, 2), dtype=np.int32)
        return np.ctypeslib.as_array(ptr, shape=(n, 2)).copy()

    ngrids = property(lambda self: _lib().MultiGrid_get_ngrids(self._this))
    nspecies = property(lambda self: _lib().MultiGrid_get_nspecies(self._this))

    def show(self):
        print('MultiGrid with', self.ngrids, 'grids')


# -------------------------------------------------------------- extrapolations
class Extrapolation(object):
    def eval_left(self, x):
        return _lib().Extrapolation_eval_left(self._this, x)

    def eval_right(self, x):
        return _lib().Extrapolation_eval_right(self._this, x)

    def deriv_left(self, x):
        return _lib().Extrapolation_deriv_left(self._this, x)

    def deriv_right(self, x):
        return _lib().Extrapolation_deriv_right(self._this, x)

    def has_tail(self):
        return _lib().Extrapolation_has_tail(self._this)

    def to_string(self):
        return self.__class__.__name__


class ZeroExtrapolation(Extrapolation):
    def __init__(self):
        self._this = _lib().ZeroExtrapolation_new()


class CuspExtrapolation(Extrapolation):
    """a exp(b (x - x0)) below the first point, zero above the last."""

    def __init__(self):
        self._this = _lib().CuspExtrapolation_new()


class PowerExtrapolation(Extrapolation):
    """a x^power above the last point."""

    def __init__(self, power):
        self._this = _lib().PowerExtrapolation_new(power)
        self._power = _lib().PowerExtrapolation_get_power(self._this)

    def to_string(self):
        return 'PowerExtrapolation %s' % repr(self.power)

    power = property(lambda self: self._power)


class PotentialExtrapolation(Extrapolation):
    """r^l below the first point and r^-(l+1) above the last (Poisson solutions)."""

    def __init__(self, l):
        self.l = l
        self._this = _lib().PotentialExtrapolation_new(l)
        if not self._this:
            check()

    def to_string(self):
        return 'PotentialExtrapolation %s' % repr(self.l)


class CubicSpline(object):
    """Cubic spline on a radial transform's uniform t-axis (cubic_spline.py:16-140).

    With ``dx`` omitted the t-derivatives solve the continuous-second-
    derivative system.
    """

    def __init__(self, y, dx=None, rtransform=None, extrapolation=None, v=None):
        self._y = np.ascontiguousarray(y, dtype=np.float64)
        n = self._y.shape[0]
        self._rtransform = IndentityRadialTransform(n) if rtransform is None else rtransform
        if v is None:
            v = self._rtransform.deriv_all()
        if dx is None:
            self._dt = np.zeros(n, np.float64)
            _lib().solve_cubic_spline_system(self._y, self._dt, n)
            self._dx = self._dt / v
        else:
            self._dx = np.ascontiguousarray(dx, dtype=np.float64)
            self._dt = np.ascontiguousarray(self._dx * v)
        self._extrapolation = CuspExtrapolation() if extrapolation is None else extrapolation
        self._this = _lib().CubicSpline_new(self._y, self._dt, self._extrapolation._this,
                                            self._rtransform._this, n)
        if not self._this:
            check()

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().CubicSpline_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def __call__(self, new_x, new_y=None):
        new_x = np.ascontiguousarray(new_x, dtype=np.float64)
        if new_y is None:
            new_y = np.zeros(new_x.shape[0], np.float64)
        _lib().CubicSpline_eval(self._this, new_x, new_y, new_x.shape[0])
        return new_y

    def deriv(self, new_x, new_dx=None):
        new_x = np.ascontiguousarray(new_x, dtype=np.float64)
        if new_dx is None:
            new_dx = np.zeros(new_x.shape[0], np.float64)
        _lib().CubicSpline_eval_deriv(self._this, new_x, new_dx, new_x.shape[0])
        return new_dx

    y = property(lambda self: self._y)
    dx = property(lambda self: self._dx)
    dt = property(lambda self: self._dt)
    first_x = property(lambda self: _lib().CubicSpline_get_first_x(self._this))
    last_x = property(lambda self: _lib().CubicSpline_get_last_x(self._this))
    extrapolation = property(lambda self: self._extrapolation)
    rtransform = property(lambda self: self._rtransform)


# --------------------------------------------------------------------- Poisson
def _torch():
    import torch
    if not torch.cuda.is_available():
        raise NapmoError('a CUDA device is required for the grid Poisson solver')
    return torch


def coulomb_potential_device(grid, rho_dev, lmax, v_dev, accumulate=False, stream=None,
                             raw=None):
    """Device Poisson solve: v = V_H[rho] at the grid points (torch tensors)."""
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    ry = rd = None
    if raw is not None:
        ry, rd = raw
    checked(_lib().napmo_gpu_poisson(grid._this, rho_dev.data_ptr(), int(lmax), v_dev.data_ptr(),
                                     1 if accumulate else 0,
                                     ry.data_ptr() if ry is not None else None,
                                     rd.data_ptr() if rd is not None else None, stream))


def poisson_solver(grid, _dens, lmax, sph_exp=None):
    """Spherically expanded potential U[atom][lm] as CubicSplines (poisson_solver.py:18-118).

    Projection, spline and Hermite-FEM radial solves run on the GPU.
    """
    if sph_exp is not None:
        raise NapmoError('precomputed expansions are not accepted; pass the density')
    torch = _torch()
    dens = torch.as_tensor(np.ascontiguousarray(_dens, dtype=np.float64), device='cuda')
    v = torch.empty(grid.size, dtype=torch.float64, device='cuda')
    nraw = _lib().napmo_poisson_raw_size(grid._this, int(lmax))
    ry = torch.empty(nraw, dtype=torch.float64, device='cuda')
    rd = torch.empty(nraw, dtype=torch.float64, device='cuda')
    coulomb_potential_device(grid, dens, lmax, v, raw=(ry, rd))
    torch.cuda.current_stream().synchronize()
    ry, rd = ry.cpu().numpy(), rd.cpu().numpy()
    lsize = (lmax + 1) ** 2
    U, off = [], 0
    for atgrid in grid.atgrids:
        rgrid = atgrid.radial_grid
        n = rgrid.size
        rtf = rgrid.rtransform
        j1 = rtf.deriv_all()
        res = []
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                idx = l * l + (m + l)
                y = ry[off + idx * n: off + (idx + 1) * n].copy()
                dt = rd[off + idx * n: off + (idx + 1) * n].copy()
                res.append(CubicSpline(y, dt / j1, rtf, PotentialExtrapolation(l), v=j1))
        off += lsize * n
        U.append(res)
    return U


def solve_ode2(b, a, f, bcs, extrapolation=None, j1=None, j2=None, j3=None):
    """Second-order ODE u'' + b u' + a u = f by Hermite finite elements (ode2.py:35-118).

    The FEM matrix is assembled exactly as nAPMO does (build_ode2) and solved
    with a dense LU; this utility serves single ODEs from Python, while the
    Poisson pipeline solves its systems in batches on the GPU.
    """
    rtf = b.rtransform
    if rtf.to_string() != a.rtransform.to_string():
        raise ValueError('The RTransform objects of b and a do not match.')
    if rtf.to_string() != f.rtransform.to_string():
        raise ValueError('The RTransform objects of b and f do not match.')
    j1 = rtf.deriv_all() if j1 is None else j1
    j2 = rtf.deriv2_all() if j2 is None else j2
    j3 = rtf.deriv3_all() if j3 is None else j3
    j1sq = j1 * j1
    by_new = j1 * b.y - j2 / j1
    bd_new = j2 * b.y + j1sq * b.dx + (j2 * j2 - j1 * j3) / j1sq
    ay_new = a.y * j1sq
    ad_new = (a.dx * j1sq + 2 * a.y * j2) * j1
    fy_new = f.y * j1sq
    fd_new = (f.dx * j1sq + 2 * f.y * j2) * j1
    new_bcs = (bcs[0], None if bcs[1] is None else bcs[1] * j1[0],
               bcs[2], None if bcs[3] is None else bcs[3] * j1[-1])
    npoint = by_new.shape[0]

    def merge(y, d):
        return np.ascontiguousarray(np.array([y, d]).T.ravel())

    c_bcs = np.array([np.nan if x is None else x for x in new_bcs], dtype=np.float64)
    coeffs = np.zeros((2 * npoint, 2 * npoint), dtype=np.float64)
    rhs = np.zeros(2 * npoint, dtype=np.float64)
    _lib().build_ode2(merge(by_new, bd_new), merge(ay_new, ad_new), merge(fy_new, fd_new),
                      c_bcs, coeffs, rhs, npoint)
    import scipy.linalg
    solution = scipy.linalg.solve(coeffs, rhs)
    return CubicSpline(solution[::2].copy(), solution[1::2] / j1, rtf, extrapolation)
