"""Local functionals on the grid (``napmo.functional``), on the device.

``Functional`` mirrors nAPMO's electronic functional object
(napmo/functional/xc_interface.py:14-133): 'lda' = Dirac-Slater exchange plus
VWN5 correlation, unpolarised, with compute_exchange / compute_correlation
returning (zk, vrho) like pylibxc (arrays of shape (n, 1); energies per
particle).  nAPMO computes them through LibXC; here the published forms run
in napmo_gpu_lda_xc.  ``epc17_2`` and ``isc_functional_selector`` mirror
napmo/functional/interspecies_correlation.py:12-68 (napmo_gpu_epc17_2).
Inputs may be numpy arrays (results come back as numpy) or CUDA tensors
(results stay on the device).
"""
import numpy as np

from . import cext
from .cext import NapmoError, checked


def _torch():
    import torch
    return torch


def _device(x):
    """(device tensor, was the input a numpy array)."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        return x.to(device='cuda', dtype=torch.float64).contiguous().reshape(-1), False
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64).reshape(-1),
                           device='cuda'), True


def _out(t, host, shape):
    t = t.reshape(shape)
    return t.cpu().numpy() if host else t


def _stream():
    return _torch().cuda.current_stream().cuda_stream


class Functional(object):
    """Electronic exchange-correlation functional of species ``symbol``.

    Args:
        symbol (str): species symbol ('e-').
        options (dict): {'functional': {'e-': 'lda'}} (the only database entry
            of nAPMO: lda_x + lda_c_vwn); 'spin': 'unpolarized'.
    """

    _database = {'lda': {'correlation': 'lda_c_vwn', 'exchange': 'lda_x'}}

    def __init__(self, symbol, options={'functional': {'e-': 'lda'}}):
        self.options = {'correlation': 'lda_c_vwn', 'exchange': 'lda_x', 'spin': 'unpolarized'}
        self.options.update(options)
        name = options.get('functional', {}).get('e-', 'lda')
        if name not in self._database:
            raise NotImplementedError(str(name) + ' Functional NOT available!')
        self.options.update(self._database[name])
        if self.options['spin'] != 'unpolarized':
            raise NotImplementedError('only the unpolarised LDA is available')
        self._symbol = symbol
        self._x_factor = 0.0

    def _compute(self, rho, which):
        torch = _torch()
        r, host = _device(rho)
        n = r.numel()
        zk = torch.empty(n, dtype=torch.float64, device='cuda')
        vrho = torch.empty_like(zk)
        args = [zk.data_ptr(), vrho.data_ptr(), None, None] if which == 'x' else \
            [None, None, zk.data_ptr(), vrho.data_ptr()]
        checked(cext.lib.napmo_gpu_lda_xc(n, r.data_ptr(), *args, _stream()))
        return _out(zk, host, (n, 1)), _out(vrho, host, (n, 1))

    def compute_correlation(self, rho):
        """(zk, vrho) of VWN5 correlation at every density value."""
        return self._compute(rho, 'c')

    def compute_exchange(self, rho):
        """(zk, vrho) of Dirac-Slater exchange at every density value."""
        return self._compute(rho, 'x')

    def show(self):
        print("\nFunctional Information:", self.symbol)
        print("-" * (24 + len(self.symbol)))
        print(self.options)

    symbol = property(lambda self: self._symbol)
    correlation = property(lambda self: self.options.get('correlation'))
    exchange = property(lambda self: self.options.get('exchange'))
    spin = property(lambda self: self.options.get('spin'))
    x_factor = property(lambda self: self._x_factor)


def epc17_2(rhoE, rhoN):
    """(energy per electron, electron potential, nuclear potential) of the
    epc17-2 electron-proton correlation at common points."""
    torch = _torch()
    e, host = _device(rhoE)
    q, _ = _device(rhoN)
    if e.numel() != q.numel():
        raise NapmoError('rhoE and rhoN must hold the same points')
    n = e.numel()
    ene, pe, pn = (torch.empty(n, dtype=torch.float64, device='cuda') for _ in range(3))
    checked(cext.lib.napmo_gpu_epc17_2(n, e.data_ptr(), q.data_ptr(), ene.data_ptr(),
                                       pe.data_ptr(), pn.data_ptr(), _stream()))
    return tuple(_out(t, host, (n,)) for t in (ene, pe, pn))


def isc_functional_selector(name):
    """The interspecies functional called ``name`` (None for None)."""
    if name is None:
        return None
    assert isinstance(name, str)
    functional = {'epc17-2': epc17_2}.get(name)
    if functional is None:
        raise NotImplementedError(name + " Functional NOT available!")
    return functional
