"""ctypes bindings of ``libnapmo.so`` (built by ``napmo_b200.build``).

The nAPMO-compatible symbols carry the argument types nAPMO declares in
``napmo/__init__.py:95-585``; the device-pointer entry points (``napmo_gpu_*``,
``napmo_fock_plan_*``) are this library's own.  Loading fails loudly when the
library is missing: there is no Python fallback for any of it.
"""
import ctypes
import os
from ctypes import (POINTER, c_bool, c_char_p, c_double, c_int, c_long,
                    c_void_p)

import numpy as np
import numpy.ctypeslib as npct

LIBPATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'lib', 'libnapmo.so')


class NapmoError(RuntimeError):
    """Raised when a libnapmo entry point reports an error."""


def _load():
    if not os.path.exists(LIBPATH):
        raise ImportError('libnapmo.so is not built (%s); run `python napmo_b200/build.py`'
                          % LIBPATH)
    return ctypes.CDLL(LIBPATH)


lib = _load()

a1df = npct.ndpointer(dtype=np.double, ndim=1, flags='CONTIGUOUS')
a2df = npct.ndpointer(dtype=np.double, ndim=2, flags='CONTIGUOUS')
a3df = npct.ndpointer(dtype=np.double, ndim=3, flags='CONTIGUOUS')
a1di = npct.ndpointer(dtype=np.int32, ndim=1, flags='CONTIGUOUS')
a1dli = npct.ndpointer(dtype=np.int64, ndim=1, flags='CONTIGUOUS')
aptr = npct.ndpointer(c_void_p, flags='C_CONTIGUOUS')
PD = POINTER(c_double)


def _sig(name, restype, argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


_SIGS = [
    # errors / memory
    ('napmo_last_error', c_int, [c_char_p, c_int]),
    ('napmo_free_array', None, [c_void_p]),
    # wavefunction
    ('wavefunction_guess_hcore', None, [c_void_p]),
    ('wavefunction_transformation_matrix', None, [c_void_p]),
    ('wavefunction_compute_coefficients', None, [c_void_p]),
    ('wavefunction_compute_density', None, [c_void_p]),
    ('wavefunction_compute_energy', None, [c_void_p]),
    ('wavefunction_iterate', None, [c_void_p]),
    ('nwavefunction_compute_density_from_dm', None,
     [c_void_p, c_void_p, a2df, a1df, c_double, a1df]),
    ('nwavefunction_compute_2body_matrix', None, [c_void_p, c_void_p, a2df, a1df, a2df]),
    ('nwavefunction_compute_coupling', None, [c_void_p, c_void_p, a2df, a1df, a2df]),
    ('nwavefunction_compute_xc_matrix', None, [c_void_p, c_void_p, a2df, a1df]),
    # gaussians
    ('PrimitiveGaussian_new', c_void_p, [a1di, a1df, c_double, c_double]),
    ('PrimitiveGaussian_del', None, [c_void_p]),
    ('PrimitiveGaussian_compute', None, [c_void_p, a2df, a1df, c_int]),
    ('PrimitiveGaussian_deriv', None, [c_void_p, a2df, a2df, c_int]),
    ('PrimitiveGaussian_overlap', c_double, [c_void_p, c_void_p]),
    ('PrimitiveGaussian_get_l', None, [c_void_p, a1di]),
    ('PrimitiveGaussian_get_origin', None, [c_void_p, a1df]),
    ('PrimitiveGaussian_get_zeta', c_double, [c_void_p]),
    ('PrimitiveGaussian_get_coeff', c_double, [c_void_p]),
    ('PrimitiveGaussian_get_norma', c_double, [c_void_p]),
    ('ContractedGaussian_new', c_void_p, [aptr, c_int]),
    ('ContractedGaussian_del', None, [c_void_p]),
    ('ContractedGaussian_get_nprim', c_int, [c_void_p]),
    ('ContractedGaussian_get_l', None, [c_void_p, a1di]),
    ('ContractedGaussian_get_origin', None, [c_void_p, a1df]),
    ('ContractedGaussian_compute', None, [c_void_p, a2df, a1df, c_int]),
    ('ContractedGaussian_deriv', None, [c_void_p, a2df, a2df, c_int]),
    ('ContractedGaussian_overlap', c_double, [c_void_p, c_void_p]),
    ('ContractedGaussian_get_norma', c_double, [c_void_p]),
    ('BasisSet_new_empty', c_void_p, []),
    ('BasisSet_new', c_void_p, [aptr, c_int]),
    ('BasisSet_del', None, [c_void_p]),
    ('BasisSet_compute', None, [c_void_p, a2df, a2df, c_int]),
    ('BasisSet_deriv', None, [c_void_p, a2df, a3df, c_int]),
    ('BasisSet_update', None, [c_void_p, c_void_p]),
    ('BasisSet_get_nbasis', c_int, [c_void_p]),
    ('BasisSet_get_max_l', c_int, [c_void_p]),
    ('BasisSet_get_max_nprim', c_int, [c_void_p]),
    # grids
    ('AngularGrid_new', c_void_p, [c_int]),
    ('AngularGrid_del', None, [c_void_p]),
    ('AngularGrid_spherical', None, [c_void_p]),
    ('AngularGrid_integrate', c_double, [c_void_p, c_int, a1df, c_void_p]),
    ('AngularGrid_get_lorder', c_int, [c_void_p]),
    ('AngularGrid_get_points', PD, [c_void_p]),
    ('AngularGrid_get_weights', PD, [c_void_p]),
    ('RadialGrid_new', c_void_p, [c_void_p, c_double]),
    ('RadialGrid_del', None, [c_void_p]),
    ('RadialGrid_integrate', c_double, [c_void_p, c_int, a1df]),
    ('RadialGrid_deriv2', PD, [c_void_p, a1df]),
    ('RadialGrid_get_size', c_int, [c_void_p]),
    ('RadialGrid_get_radii', c_double, [c_void_p]),
    ('RadialGrid_get_points', PD, [c_void_p]),
    ('RadialGrid_get_weights', PD, [c_void_p]),
    ('AtomicGrid_new', c_void_p, [c_void_p, c_void_p, a1df]),
    ('AtomicGrid_del', None, [c_void_p]),
    ('AtomicGrid_integrate', PD, [c_void_p, c_int, c_int, c_int, a1df]),
    ('AtomicGrid_spherical_expansion', PD, [c_void_p, a1df, c_int]),
    ('AtomicGrid_get_size', c_int, [c_void_p]),
    ('AtomicGrid_get_radii', c_double, [c_void_p]),
    ('AtomicGrid_get_origin', PD, [c_void_p]),
    ('AtomicGrid_get_points', PD, [c_void_p]),
    ('AtomicGrid_get_weights', PD, [c_void_p]),
    ('BeckeGrid_new', c_void_p, [aptr, c_int, c_int, c_double]),
    ('BeckeGrid_del', None, [c_void_p]),
    ('BeckeGrid_from_points', c_void_p, [a2df, c_int, c_int]),
    ('BeckeGrid_integrate', c_double, [c_void_p, a1df]),
    ('BeckeGrid_get_ncenter', c_int, [c_void_p]),
    ('BeckeGrid_get_size', c_int, [c_void_p]),
    ('BeckeGrid_get_radii', PD, [c_void_p]),
    ('BeckeGrid_get_points', PD, [c_void_p]),
    ('BeckeGrid_get_weights', PD, [c_void_p]),
    ('BeckeGrid_get_origin', PD, [c_void_p]),
    ('BeckeGrid_get_becke_weights', PD, [c_void_p]),
    ('eval_decomposition_grid', None, [aptr, a1df, a1df, a2df, c_void_p, c_long, c_long]),
    ('MultiGrid_new', c_void_p, [c_int]),
    ('MultiGrid_del', None, [c_void_p]),
    ('MultiGrid_get_common_index', POINTER(c_int), [c_void_p, c_int, c_int]),
    ('MultiGrid_get_common_index_size', c_int, [c_void_p, c_int, c_int]),
    ('MultiGrid_get_ngrids', c_int, [c_void_p]),
    ('MultiGrid_get_nspecies', c_int, [c_void_p]),
    ('MultiGrid_add_grid', c_int, [c_void_p, c_void_p]),
    # splines / extrapolation / transforms
    ('CubicSpline_new', c_void_p, [a1df, a1df, c_void_p, c_void_p, c_int]),
    ('CubicSpline_del', None, [c_void_p]),
    ('CubicSpline_eval', None, [c_void_p, a1df, a1df, c_int]),
    ('CubicSpline_eval_deriv', None, [c_void_p, a1df, a1df, c_int]),
    ('CubicSpline_get_first_x', c_double, [c_void_p]),
    ('CubicSpline_get_last_x', c_double, [c_void_p]),
    ('CubicSpline_get_rtransform', c_void_p, [c_void_p]),
    ('CubicSpline_get_extrapolation', c_void_p, [c_void_p]),
    ('solve_cubic_spline_system', None, [a1df, a1df, c_int]),
    ('compute_cubic_spline_int_weights', None, [a1df, c_int]),
    ('Extrapolation_prepare', None, [c_void_p, c_void_p]),
    ('Extrapolation_del', None, [c_void_p]),
    ('Extrapolation_eval_left', c_double, [c_void_p, c_double]),
    ('Extrapolation_eval_right', c_double, [c_void_p, c_double]),
    ('Extrapolation_deriv_left', c_double, [c_void_p, c_double]),
    ('Extrapolation_deriv_right', c_double, [c_void_p, c_double]),
    ('Extrapolation_has_tail', c_bool, [c_void_p]),
    ('ZeroExtrapolation_new', c_void_p, []),
    ('CuspExtrapolation_new', c_void_p, []),
    ('PowerExtrapolation_new', c_void_p, [c_double]),
    ('PowerExtrapolation_get_power', c_double, [c_void_p]),
    ('PotentialExtrapolation_new', c_void_p, [c_int]),
    ('RTransform_get_npoint', c_int, [c_void_p]),
    ('RTransform_del', None, [c_void_p]),
    ('RTransform_radius', c_double, [c_void_p, c_double]),
    ('RTransform_deriv', c_double, [c_void_p, c_double]),
    ('RTransform_deriv2', c_double, [c_void_p, c_double]),
    ('RTransform_deriv3', c_double, [c_void_p, c_double]),
    ('RTransform_inv', c_double, [c_void_p, c_double]),
    ('RTransform_radius_array', None, [c_void_p, a1df, a1df, c_int]),
    ('RTransform_deriv_array', None, [c_void_p, a1df, a1df, c_int]),
    ('RTransform_deriv2_array', None, [c_void_p, a1df, a1df, c_int]),
    ('RTransform_deriv3_array', None, [c_void_p, a1df, a1df, c_int]),
    ('RTransform_inv_array', None, [c_void_p, a1df, a1df, c_int]),
    ('IdentityRTransform_new', c_void_p, [c_int]),
    ('PowerRTransform_new', c_void_p, [c_double, c_double, c_int]),
    ('PowerRTransform_get_rmin', c_double, [c_void_p]),
    ('PowerRTransform_get_rmax', c_double, [c_void_p]),
    ('PowerRTransform_get_power', c_double, [c_void_p]),
    ('ChebyshevRTransform_new', c_void_p, [c_double, c_int]),
    ('ChebyshevRTransform_get_radii', c_double, [c_void_p]),
    ('Cell_new', c_void_p, [c_void_p, c_int]),
    ('Cell_del', None, [c_void_p]),
    ('build_ode2', None, [a1df, a1df, a1df, a1df, a2df, a1df, c_long]),
    ('dot_multi_moments', None,
     [c_long, c_long, a1df, a2df, a1df, c_long, c_long, a1dli, a2df, c_long]),
    # device API
    ('napmo_grid_device_arrays', c_int,
     [c_void_p, POINTER(c_void_p), POINTER(c_void_p), POINTER(c_void_p), POINTER(c_void_p),
      POINTER(c_void_p)]),
    ('napmo_gpu_becke_weights', c_int,
     [c_int, c_int, c_void_p, c_void_p, c_void_p, a1df, a1df, a1di, c_void_p, c_void_p]),
    ('napmo_gpu_basis_values', c_int,
     [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_long, c_void_p, c_void_p]),
    ('napmo_gpu_density', c_int, [c_int, c_int, c_void_p, c_long, c_void_p, c_void_p, c_void_p]),
    ('napmo_gpu_quadrature', c_int,
     [c_int, c_int, c_void_p, c_void_p, c_long, c_void_p, c_void_p, c_void_p]),
    ('napmo_gpu_combine_weights', c_int,
     [c_int, c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_gpu_poisson', c_int,
     [c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    ('napmo_poisson_raw_size', c_long, [c_void_p, c_int]),
    ('napmo_grid_set_poisson_tolerance', c_int, [c_void_p, c_double]),
    ('napmo_gpu_lda_xc', c_int,
     [c_long, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_gpu_lda_xc_polarized', c_int,
     [c_long, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
      c_void_p]),
    ('napmo_gpu_epc17_2', c_int,
     [c_long, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_gpu_kinetic', c_int,
     [c_void_p, c_int, c_int, c_void_p, c_long, c_double, c_void_p, c_void_p]),
    ('napmo_gpu_dpsi', c_int,
     [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_long, a1df, a1df, c_double,
      c_void_p, c_void_p]),
    ('napmo_gpu_operator_matrix', c_int,
     [c_void_p, c_int, c_int, c_void_p, c_long, c_void_p, c_long, c_void_p, c_void_p]),
    ('napmo_gpu_one_body', c_int,
     [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('LibintInterface_new', c_void_p, [c_int]),
    ('LibintInterface_del', None, [c_void_p]),
    ('LibintInterface_add_basis', None, [c_void_p, c_void_p]),
    ('LibintInterface_add_pointcharges', None, [c_void_p, c_int, a1df]),
    ('LibintInterface_get_nbasis', c_int, [c_void_p]),
    ('LibintInterface_compute_1body_ints', None, [c_void_p, c_int, a2df]),
    ('napmo_gpu_nuclear_potential', c_int,
     [c_int, c_void_p, c_void_p, c_void_p, c_int, a2df, c_void_p, c_void_p]),
    ('napmo_fock_plan_new', c_void_p, [c_void_p, c_void_p, c_int, c_void_p]),
    ('napmo_fock_plan_free', None, [c_void_p]),
    ('napmo_fock_plan_refresh', c_int, [c_void_p, c_void_p]),
    ('napmo_grid_set_centers', c_int, [c_void_p, a2df]),
    ('napmo_fock_plan_info', c_int,
     [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_long), POINTER(c_void_p)]),
    ('napmo_fock_plan_density', c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_fock_plan_quadrature', c_int,
     [c_void_p, c_double, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_fock_plan_build', c_int,
     [c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_fock_plan_build_host', c_int,
     [c_void_p, a2df, c_double, c_void_p, a2df, c_void_p]),
    ('napmo_fock_plan_set_precision', c_int, [c_void_p, c_int]),
    ('napmo_fock_plan_set_poisson_tolerance', c_int, [c_void_p, c_double]),
    ('napmo_fock_plan_poisson', c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_fock_plan_poisson_many', c_int, [c_void_p, c_int, c_void_p, c_long, c_void_p,
                                             c_void_p]),
    ('napmo_gpu_poisson_many', c_int, [c_void_p, c_int, c_void_p, c_long, c_int, c_void_p,
                                       c_void_p]),
    ('napmo_fock_plan_screening', c_int, [c_void_p, POINTER(c_void_p), POINTER(c_int)]),
    ('napmo_fock_plan_set_fp64_screening', c_int, [c_void_p, c_double, c_void_p]),
    ('napmo_fock_plan_int8_bytes', c_long, [c_void_p]),
    ('napmo_fock_plan_release_phi', c_int, [c_void_p]),
    ('napmo_fock_batch_new', c_void_p, [c_void_p, c_int, c_double]),
    ('napmo_fock_batch_free', None, [c_void_p]),
    ('napmo_fock_batch_buffers', c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    ('napmo_fock_batch_build', c_int, [c_void_p, c_void_p]),
    ('napmo_fock_batch_tune', c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    ('napmo_fock_batch_config', c_int, [c_void_p, c_void_p, c_void_p]),
    ('napmo_fock_batch_set_mode', c_int, [c_void_p, c_int]),
    ('napmo_fock_batch_queue_selftest', c_int, [c_void_p, c_double, c_void_p, c_void_p]),
    ('napmo_fock_batch_status', c_int, [c_void_p, c_void_p, c_void_p]),
    ('napmo_basis_one_body', c_int, [c_void_p, a2df, a2df]),
    ('napmo_basis_get_origins', c_int, [c_void_p, a2df]),
    ('napmo_basis_set_origins', c_int, [c_void_p, a2df]),
    ('napmo_grid_energy_gradient', c_int,
     [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('napmo_tc_status', c_int, [c_void_p, c_int]),
    ('napmo_tc_wait_selftest', c_int, [c_void_p, c_void_p]),
    ('napmo_gpu_quadrature_noalloc', c_int,
     [c_int, c_int, c_void_p, c_void_p, c_long, c_void_p, c_void_p, c_void_p]),
]

for _name, _res, _args in _SIGS:
    _sig(_name, _res, _args)


def last_error():
    buf = ctypes.create_string_buffer(1024)
    code = lib.napmo_last_error(buf, 1024)
    return code, buf.value.decode(errors='replace')


def check(result=None):
    """Raise NapmoError if the last libnapmo call on this thread failed."""
    code, msg = last_error()
    if code != 0:
        raise NapmoError('libnapmo error %d: %s' % (code, msg))
    return result


def checked(status):
    """Raise for a nonzero status returned by an int entry point."""
    if status != 0:
        code, msg = last_error()
        raise NapmoError('libnapmo error %d: %s' % (status, msg))
    return status


def as_array(ptr, shape):
    if not ptr:
        check()
        raise NapmoError('libnapmo returned a null pointer')
    return np.ctypeslib.as_array(ptr, shape=shape)
