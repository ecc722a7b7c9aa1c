"""Device-resident grid Fock builds (the hot path), driven through the C-ABI.

A ``FockBuilder`` evaluates the basis on the grid once (phi stays in HBM for
the whole SCF) and then, per build, runs on one CUDA stream:

  rho = diag(phi^T D phi)                  (FP64 DFMA GEMM, fused epilogue)
  v   = q V_H[rho]                         (Becke-Dickson Poisson on device)
  F   = phi diag(wb w (v + v_ext)) phi^T   (FP64 split-K GEMM)

torch provides device memory and the stream; every byte of arithmetic is in
libnapmo's kernels.  Reference call stack: napmo/wavefunction/psi_hybrid.py:
81-110 (coupling), napmo/wavefunction/ntwobody.py:15-46 (Coulomb potential),
src/wavefunction/nwavefunction.cpp:77-107,161-197 (quadratures).
"""
from ctypes import byref, c_double, c_int, c_long, c_void_p

import numpy as np

from . import cext
from .cext import checked, NapmoError


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise NapmoError('FockBuilder needs a CUDA device')
    return torch


def _stream(torch, stream):
    return (stream or torch.cuda.current_stream()).cuda_stream


class FockBuilder(object):
    """Grid Fock builds for one species (basis) on one molecular grid.

    Args:
        grid (BeckeGrid): molecular grid (Becke weights already on device).
        basis (BasisSet): basis of the species.
        lmax (int or 'per-atom'): angular cutoff of the Poisson expansion;
            nAPMO uses lebedev_get_order(nang) // 2 (psi_numeric.py:66).
            'per-atom': each atom's own Lebedev rule (uneven grids).  -1: no
            Poisson tables (quadratures only).
    """

    PRECISIONS = {'fp64': 0, 'int8x4': 1}

    def __init__(self, grid, basis, lmax, stream=None, precision='fp64'):
        torch = _torch()
        self.torch = torch
        self.grid = grid
        self.basis = basis
        self.lmax = -2 if lmax == 'per-atom' else int(lmax)
        self._plan = cext.lib.napmo_fock_plan_new(grid._this, basis._this, self.lmax,
                                                  _stream(torch, stream))
        if not self._plan:
            cext.check()
            raise NapmoError('fock plan construction failed')
        n, npt, ld, phi = c_int(), c_int(), c_long(), c_void_p()
        checked(cext.lib.napmo_fock_plan_info(self._plan, byref(n), byref(npt), byref(ld),
                                              byref(phi)))
        self.n, self.npoint, self.ld = n.value, npt.value, ld.value
        self.set_precision(precision)

    def set_precision(self, precision, poisson_tol=None):
        """'fp64' (CUDA cores) or 'int8x4' (int8 slices on the tensor cores) for
        rho and F; the Poisson solve is FP64 in both.  The Poisson truncation
        tolerance follows the mode (0: every (l, m) as nAPMO; 1e-9 a.u. for
        'int8x4') unless `poisson_tol` is given."""
        checked(cext.lib.napmo_fock_plan_set_precision(self._plan, self.PRECISIONS[precision]))
        self.precision = precision
        if poisson_tol is not None:
            self.set_poisson_tolerance(poisson_tol)

    def set_fp64_screening(self, tol=1e-24, stream=None):
        """FP64 mode: skip the points with |wb w| max_mu phi_mu(p)^2 < tol in
        the density, the potential evaluation and the quadrature (the int8
        mode's screening, 1e-24 by default); 0 restores every point."""
        checked(cext.lib.napmo_fock_plan_set_fp64_screening(self._plan, float(tol),
                                                            _stream(self.torch, stream)))

    def set_poisson_tolerance(self, tol):
        """Truncation tolerance (a.u.) of the potential evaluation: per atom and
        radial interval, l-blocks whose bounded contribution to any point sums
        to at most `tol` are skipped (0: none)."""
        checked(cext.lib.napmo_fock_plan_set_poisson_tolerance(self._plan, float(tol)))

    def kept_points(self):
        """Boolean tensor of the grid points the current mode uses, or None
        when it uses all ('int8x4' screens out the points with
        |w_becke w| max_mu phi_mu^2 < 1e-24; rho and v are 0 there)."""
        keep, nkeep = c_void_p(), c_int()
        checked(cext.lib.napmo_fock_plan_screening(self._plan, byref(keep), byref(nkeep)))
        if not keep.value:
            return None
        return _view(self.torch, keep.value, (self.npoint,), '<i4') != 0

    def refresh(self, stream=None):
        """Re-evaluates the basis on the grid after either moved
        (BeckeGrid.set_centers, BasisSet.set_origins), in the plan's buffers."""
        checked(cext.lib.napmo_fock_plan_refresh(self._plan, _stream(self.torch, stream)))

    def tc_status(self, reset=True, stream=None):
        """Error word of the tensor-core kernels (0: none); synchronises the stream."""
        return cext.lib.napmo_tc_status(_stream(self.torch, stream), 1 if reset else 0)

    def __del__(self):
        if getattr(self, '_plan', None):
            try:
                cext.lib.napmo_fock_plan_free(self._plan)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._plan = None

    def _dev(self, x, shape=None):
        t = self.torch
        if x is None:
            return None
        if not isinstance(x, t.Tensor):
            x = t.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device='cuda')
        x = x.to(device='cuda', dtype=t.float64).contiguous()
        if shape is not None and tuple(x.shape) != tuple(shape):
            raise ValueError('expected shape %s, got %s' % (shape, tuple(x.shape)))
        return x

    def density(self, D, stream=None):
        """rho at every grid point for density matrix D (n x n, symmetric)."""
        t = self.torch
        D = self._dev(D, (self.n, self.n))
        rho = t.empty(self.npoint, dtype=t.float64, device='cuda')
        checked(cext.lib.napmo_fock_plan_density(self._plan, D.data_ptr(), rho.data_ptr(),
                                                 _stream(t, stream)))
        return rho

    def quadrature(self, q=1.0, v=None, vext=None, stream=None):
        """F = phi diag(wb w (q v + vext)) phi^T for grid potentials v, vext."""
        t = self.torch
        v = self._dev(v, (self.npoint,))
        vext = self._dev(vext, (self.npoint,))
        F = t.empty((self.n, self.n), dtype=t.float64, device='cuda')
        checked(cext.lib.napmo_fock_plan_quadrature(
            self._plan, float(q), v.data_ptr() if v is not None else None,
            vext.data_ptr() if vext is not None else None, F.data_ptr(), _stream(t, stream)))
        return F

    def coulomb_potential(self, rho, stream=None):
        """V_H[rho] at every grid point (device Poisson solve)."""
        t = self.torch
        rho = self._dev(rho, (self.npoint,))
        v = t.empty(self.npoint, dtype=t.float64, device='cuda')
        checked(cext.lib.napmo_fock_plan_poisson(self._plan, rho.data_ptr(), v.data_ptr(),
                                                 _stream(t, stream)))
        return v

    def coulomb_potentials(self, rho, stream=None):
        """V_H of every row of rho (k x npoint) in one library call."""
        t = self.torch
        rho = self._dev(rho).reshape(-1, self.npoint).contiguous()
        v = t.empty_like(rho)
        checked(cext.lib.napmo_fock_plan_poisson_many(self._plan, rho.shape[0], rho.data_ptr(),
                                                      self.npoint, v.data_ptr(),
                                                      _stream(t, stream)))
        return v

    def build(self, D, q=1.0, vext=None, stream=None, out=None):
        """One grid Fock build: returns (F, rho, v) with v = q V_H[rho]."""
        t = self.torch
        D = self._dev(D, (self.n, self.n))
        vext = self._dev(vext, (self.npoint,))
        F = out if out is not None else t.empty((self.n, self.n), dtype=t.float64, device='cuda')
        rho = t.empty(self.npoint, dtype=t.float64, device='cuda')
        v = t.empty(self.npoint, dtype=t.float64, device='cuda')
        checked(cext.lib.napmo_fock_plan_build(
            self._plan, D.data_ptr(), float(q), vext.data_ptr() if vext is not None else None,
            F.data_ptr(), rho.data_ptr(), v.data_ptr(), _stream(t, stream)))
        return F, rho, v

    def build_host(self, D, q=1.0, vext=None, stream=None):
        """Same build from/to host numpy arrays through the C-ABI (copies inside)."""
        t = self.torch
        D = np.ascontiguousarray(D, dtype=np.float64)
        F = np.empty((self.n, self.n), dtype=np.float64)
        vp = None
        if vext is not None:
            vext = np.ascontiguousarray(vext, dtype=np.float64)
            vp = vext.ctypes.data
        checked(cext.lib.napmo_fock_plan_build_host(self._plan, D, float(q), vp, F,
                                                    _stream(t, stream)))
        return F

    def phi(self):
        """phi [n][ld] on the device as a torch view (ld >= npoint, zero padded);
        evaluated again first when release_fp64_phi freed it.  The view is valid
        until the next release_fp64_phi."""
        n, npt, ld, phi = c_int(), c_int(), c_long(), c_void_p()
        checked(cext.lib.napmo_fock_plan_info(self._plan, byref(n), byref(npt), byref(ld),
                                              byref(phi)))
        return _view(self.torch, phi.value, (self.n, self.ld))

    def release_fp64_phi(self):
        """'int8x4' only: frees the FP64 phi (n x ld doubles; 7.6 GB for
        C20H42 / cc-pVDZ on 100x302 points per atom), which the int8 builds do
        not read.  FP64 builds, phi(), set_fp64_screening and refresh evaluate
        it again when they need it.  No counterpart in nAPMO."""
        checked(cext.lib.napmo_fock_plan_release_phi(self._plan))


def _view(torch, ptr, shape, typestr='<f8'):
    """A torch tensor aliasing libnapmo device memory (read-only use)."""
    n = int(np.prod(shape))

    class _Holder(object):
        __cuda_array_interface__ = {
            'shape': (n,), 'typestr': typestr, 'data': (ptr, False), 'version': 2}

    return torch.as_tensor(_Holder(), device='cuda').view(*shape)


class FockBatch(object):
    """Grid Fock builds of many molecules (FockBuilders of uneven grid and
    basis sizes) in one CUDA-graph launch.

    The batch owns a device D and F per molecule (``D(i)``, ``F(i)`` torch
    views).  ``build(Ds)`` copies the densities in (optional) and launches the
    graph; ``tune()`` runs the library's autotuner over launch shapes.

    Args:
        builders (list of FockBuilder): one per molecule (kept alive here).
        q (float): charge applied to every potential.
    """

    def __init__(self, builders, q=1.0):
        torch = _torch()
        self.torch = torch
        self.builders = list(builders)
        arr = (c_void_p * len(self.builders))(*[b._plan for b in self.builders])
        self._this = cext.lib.napmo_fock_batch_new(arr, len(self.builders), float(q))
        if not self._this:
            cext.check()
            raise NapmoError('batch construction failed')
        self._D, self._F = [], []
        for i, b in enumerate(self.builders):
            dp, fp = c_void_p(), c_void_p()
            checked(cext.lib.napmo_fock_batch_buffers(self._this, i, byref(dp), byref(fp)))
            self._D.append(_view(torch, dp.value, (b.n, b.n)))
            self._F.append(_view(torch, fp.value, (b.n, b.n)))

    def __len__(self):
        return len(self.builders)

    def D(self, i):
        return self._D[i]

    def F(self, i):
        return self._F[i]

    def build(self, Ds=None, stream=None):
        """Copies Ds (optional list of n x n arrays) into the batch and builds
        every molecule; returns the list of F views (valid until the next build)."""
        t = self.torch
        if Ds is not None:
            for dst, D in zip(self._D, Ds):
                dst.copy_(t.as_tensor(D, dtype=t.float64), non_blocking=False)
        checked(cext.lib.napmo_fock_batch_build(self._this, _stream(t, stream)))
        return self._F

    def tune(self, reps=3, stream=None):
        """Times candidate launch shapes on the batch's current densities (load
        representative ones first: the Poisson truncation of the int8 mode
        makes the cost depend on them) and keeps the fastest; returns
        {'nstream', 'budget', 'ms'}."""
        ns, bud, ms = c_int(), c_int(), c_double()
        checked(cext.lib.napmo_fock_batch_tune(self._this, _stream(self.torch, stream), int(reps),
                                               byref(ns), byref(bud), byref(ms)))
        return {'nstream': ns.value, 'budget': bud.value, 'ms': ms.value}

    MODES = {'streams': 0, 'stages': 1}

    def set_mode(self, mode):
        """'streams': the molecules' own launch chains spread over capture
        streams (one graph); 'stages': one launch per stage for the whole batch
        (persistent density and quadrature launches over device work queues,
        one Poisson plan over every grid; FP64 builders)."""
        checked(cext.lib.napmo_fock_batch_set_mode(self._this, self.MODES[mode]))
        self.mode = mode

    def queue_selftest(self, timeout_s=0.2, stream=None):
        """'stages' mode: the density stage with a queue that is never posted;
        returns the queue's error word (5 when the bounded waits ran out)."""
        st = c_int()
        checked(cext.lib.napmo_fock_batch_queue_selftest(self._this, float(timeout_s),
                                                         _stream(self.torch, stream), byref(st)))
        return st.value

    def status(self, stream=None):
        """Error word of the work queues since the last call (0 or 5)."""
        st = c_int()
        checked(cext.lib.napmo_fock_batch_status(self._this, _stream(self.torch, stream),
                                                 byref(st)))
        return st.value

    def __del__(self):
        if getattr(self, '_this', None):
            try:
                cext.lib.napmo_fock_batch_free(self._this)
            except (AttributeError, TypeError):  # library already unloaded at exit
                pass
            self._this = None
