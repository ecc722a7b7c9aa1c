"""Wave-function record and grid potentials of the nAPMO-compatible API.

``WaveFunction`` is the ctypes mirror of nAPMO's ``struct wf`` (the PSIB
Structure, napmo/wavefunction/psi_base.py:18-45) so the nwavefunction_* and
wavefunction_* entry points of libnapmo can be called exactly as nAPMO does.
``compute_coulomb`` (napmo/wavefunction/ntwobody.py:15-46) and
``compute_nuclear`` (napmo/wavefunction/nnuclear.py:15-37) run on the GPU.
"""
from ctypes import POINTER, Structure, byref, c_double, c_int

import numpy as np

from . import cext
from .cext import check, checked, NapmoError


class WaveFunction(Structure):
    _fields_ = [
        ('_S', POINTER(c_double)), ('_X', POINTER(c_double)), ('_T', POINTER(c_double)),
        ('_V', POINTER(c_double)), ('_H', POINTER(c_double)), ('_C', POINTER(c_double)),
        ('_D', POINTER(c_double)), ('_L', POINTER(c_double)), ('_G', POINTER(c_double)),
        ('_J', POINTER(c_double)), ('_XC', POINTER(c_double)), ('_F', POINTER(c_double)),
        ('_O', POINTER(c_double)),
        ('nbasis', c_int), ('ndim', c_int), ('occupation', c_int),
        ('eta', c_double), ('kappa', c_double), ('x_factor', c_double),
        ('xc_energy', c_double), ('_energy', c_double), ('_rmsd', c_double),
    ]

    _MATS = ('S', 'X', 'T', 'V', 'H', 'C', 'D', 'L', 'G', 'J', 'XC', 'F')

    def __init__(self, ndim, occupation, eta=2.0, kappa=-1.0):
        super(WaveFunction, self).__init__()
        self.ndim = self.nbasis = ndim
        self.occupation = occupation
        self.eta, self.kappa = eta, kappa
        self.x_factor = kappa / eta
        self.xc_energy = 0.0
        self._arrays = {}
        for name in self._MATS:
            a = np.zeros((ndim, ndim), dtype=np.float64)
            self._arrays[name] = a
            setattr(self, '_' + name, a.ctypes.data_as(POINTER(c_double)))
        o = np.zeros(ndim, dtype=np.float64)
        self._arrays['O'] = o
        self._O = o.ctypes.data_as(POINTER(c_double))

    def __getattr__(self, name):
        arrays = object.__getattribute__(self, '_arrays')
        if name in arrays:
            return arrays[name]
        raise AttributeError(name)

    energy = property(lambda self: self._energy)
    rmsd = property(lambda self: self._rmsd)

    def iterate(self):
        cext.lib.wavefunction_iterate(byref(self))
        check()

    def guess_hcore(self):
        cext.lib.wavefunction_guess_hcore(byref(self))
        check()


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise NapmoError('a CUDA device is required')
    return torch


def compute_coulomb(grid, dens, lmax):
    """Coulomb potential of ``dens`` at the grid points (Becke-Dickson, GPU)."""
    from .grids import coulomb_potential_device
    torch = _torch()
    rho = torch.as_tensor(np.ascontiguousarray(dens, dtype=np.float64), device='cuda')
    v = torch.empty(grid.size, dtype=torch.float64, device='cuda')
    coulomb_potential_device(grid, rho, lmax, v)
    return v.cpu().numpy()


def compute_nuclear(grid, point_charges):
    """sum_A Z_A / |r - R_A| at every grid point (GPU)."""
    torch = _torch()
    q = np.array([[*np.asarray(p.get('origin'), dtype=np.float64),
                   float(p.get('atomic_number', p.get('charge')))] for p in point_charges],
                 dtype=np.float64).reshape(-1, 4)
    x, y, z, _, _ = grid.device_arrays()
    v = torch.empty(grid.size, dtype=torch.float64, device='cuda')
    checked(cext.lib.napmo_gpu_nuclear_potential(grid.size, x, y, z, q.shape[0], q,
                                                 v.data_ptr(),
                                                 torch.cuda.current_stream().cuda_stream))
    return v.cpu().numpy()
