"""Gaussian basis side of the nAPMO-compatible Python API (``napmo.gto``).

Cartesian contracted GTOs with nAPMO's normalisation and component order
(napmo/gto/basis_set.py:122-143: for each shell of angular momentum l the
components (i, k-j, j) for k = 0..l, i = l-k, j = 0..k).  Evaluation on
points runs on the GPU.
"""
import json
import os
from ctypes import c_void_p

import numpy as np

from . import cext
from .cext import check, NapmoError

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data')
with open(os.path.join(_DATA, 'basis.json')) as _f:
    BASIS_LIBRARY = json.load(_f)


def _lib():
    return cext.lib


class PrimitiveGaussian(object):
    def __init__(self, exponent=0.5, coefficient=1.0, l=np.zeros(3, dtype=np.int32),
                 origin=np.zeros(3, dtype=np.float64)):
        l = np.ascontiguousarray(l, dtype=np.int32)
        origin = np.ascontiguousarray(origin, dtype=np.float64)
        self._this = _lib().PrimitiveGaussian_new(l, origin, exponent, coefficient)

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().PrimitiveGaussian_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def overlap(self, other):
        return _lib().PrimitiveGaussian_overlap(self._this, other._this)

    def compute(self, coord):
        coord = np.ascontiguousarray(coord, dtype=np.float64)
        out = np.empty(coord.shape[0])
        _lib().PrimitiveGaussian_compute(self._this, coord, out, coord.shape[0])
        return check(out)

    def deriv(self, coord):
        coord = np.ascontiguousarray(coord, dtype=np.float64)
        out = np.empty((coord.shape[0], 3))
        _lib().PrimitiveGaussian_deriv(self._this, coord, out, coord.shape[0])
        return check(out)

    @property
    def l(self):
        out = np.zeros(3, dtype=np.int32)
        _lib().PrimitiveGaussian_get_l(self._this, out)
        return out

    @property
    def origin(self):
        out = np.zeros(3)
        _lib().PrimitiveGaussian_get_origin(self._this, out)
        return out

    exponent = property(lambda self: _lib().PrimitiveGaussian_get_zeta(self._this))
    coefficient = property(lambda self: _lib().PrimitiveGaussian_get_coeff(self._this))
    normalization = property(lambda self: _lib().PrimitiveGaussian_get_norma(self._this))


class ContractedGaussian(object):
    def __init__(self, exponents=np.array([0.5]), coefficients=np.array([1.0]),
                 origin=np.zeros(3, dtype=np.float64), l=np.zeros(3, dtype=np.int32)):
        self._primitives = [PrimitiveGaussian(e, c, l, origin)
                            for e, c in zip(exponents, coefficients)]
        ptrs = np.array([p._this for p in self._primitives], dtype=c_void_p)
        self._this = _lib().ContractedGaussian_new(ptrs, len(self._primitives))

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().ContractedGaussian_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def overlap(self, other):
        return _lib().ContractedGaussian_overlap(self._this, other._this)

    def compute(self, coord):
        coord = np.ascontiguousarray(coord, dtype=np.float64)
        out = np.empty(coord.shape[0])
        _lib().ContractedGaussian_compute(self._this, coord, out, coord.shape[0])
        return check(out)

    def deriv(self, coord):
        coord = np.ascontiguousarray(coord, dtype=np.float64)
        out = np.empty((coord.shape[0], 3))
        _lib().ContractedGaussian_deriv(self._this, coord, out, coord.shape[0])
        return check(out)

    @property
    def l(self):
        out = np.zeros(3, dtype=np.int32)
        _lib().ContractedGaussian_get_l(self._this, out)
        return out

    @property
    def origin(self):
        out = np.zeros(3)
        _lib().ContractedGaussian_get_origin(self._this, out)
        return out

    nprim = property(lambda self: _lib().ContractedGaussian_get_nprim(self._this))
    normalization = property(lambda self: _lib().ContractedGaussian_get_norma(self._this))


def shells_for(basis_name, particle):
    """[(l, exponents, coefficients), ...] of ``particle`` in ``basis_name``."""
    lib = BASIS_LIBRARY.get(basis_name.upper(), BASIS_LIBRARY.get(basis_name))
    if lib is None:
        raise ValueError('Basis %s not available' % basis_name)
    if particle not in lib:
        raise ValueError('Basis for particle ' + particle + ' not found!')
    return lib[particle]


class BasisSet(dict):
    """Basis set of one particle at one centre (or an empty set to be extended).

    ``shells`` may be given directly as [(l, exponents, coefficients), ...]
    instead of a library basis name.
    """

    def __init__(self, basis_name, particle, origin=None, shells=None):
        super(BasisSet, self).__init__()
        self['name'] = basis_name
        self['symbol'] = particle
        self['cont'] = []
        self['nbasis'] = 0
        if origin is not None:
            if shells is None:
                shells = shells_for(basis_name, particle)
            origin = np.array(origin, dtype=np.float64)
            self['cont'] = [ContractedGaussian(np.array(e, dtype=np.float64),
                                               np.array(c, dtype=np.float64), origin,
                                               np.array([i, k - j, j], dtype=np.int32))
                            for (lval, e, c) in shells
                            for k, i in enumerate(reversed(range(lval + 1)))
                            for j in range(k + 1)]
            self['nbasis'] = len(self['cont'])
            ptrs = np.array([c._this for c in self['cont']], dtype=c_void_p)
            self._this = _lib().BasisSet_new(ptrs, self['nbasis'])
        else:
            self._this = _lib().BasisSet_new_empty()

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                _lib().BasisSet_del(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None

    def update(self, other):
        self['nbasis'] += other.get('nbasis')
        self['cont'] += other.get('cont')
        _lib().BasisSet_update(self._this, other._this)

    def origins(self):
        """Centre of every basis function (nbasis x 3, bohr)."""
        out = np.zeros((self['nbasis'], 3))
        cext.checked(_lib().napmo_basis_get_origins(self._this, out))
        return out

    def set_origins(self, origins):
        """Moves the functions to new centres (nbasis x 3, bohr) in the library's
        copy (the device copy is updated in place); plans on this basis need
        FockBuilder.refresh()."""
        origins = np.ascontiguousarray(np.asarray(origins, dtype=np.float64).reshape(-1, 3))
        cext.checked(_lib().napmo_basis_set_origins(self._this, origins))

    def compute(self, coord=np.zeros([1, 3], dtype=np.float64)):
        """phi[p, mu] at points coord[p] (GPU)."""
        coord = np.ascontiguousarray(coord, dtype=np.float64)
        out = np.empty([coord.shape[0], self['nbasis']])
        _lib().BasisSet_compute(self._this, coord, out, coord.shape[0])
        return check(out)

    def deriv(self, coord=np.zeros([1, 3], dtype=np.float64)):
        """grad phi[p, mu, xyz] at points coord[p] (GPU, analytic)."""
        coord = np.ascontiguousarray(coord, dtype=np.float64)
        out = np.empty([coord.shape[0], self['nbasis'], 3])
        _lib().BasisSet_deriv(self._this, coord, out, coord.shape[0])
        return check(out)

    @property
    def lmax(self):
        return int(np.max([c.l.sum() for c in self['cont']]))
