"""Differentiable grid quadrature energy E(D, R) (torch.autograd.Function).

For one species s of a molecular system (electrons, or a quantum nucleus), the
energy of its density in the potential of the classical nuclei, evaluated by
the Becke grid quadrature of the species:

    E(D, R) = q_s sum_p w_becke(p) w(p) rho_D(r_p) sum_C Z_C / |r_p - R_C|

The grid, the Becke weights, the basis functions and the classical charges
all move with the atoms R (bohr).  Forward: the quadrature matrix
V = phi diag(w_becke w v) phi^T on the device (napmo_fock_plan_quadrature) and
E = sum D V.  Backward: dE/dD = V, and dE/dR from the hand-written gradient
kernel (napmo_grid_energy_gradient: Becke cell-function derivatives, basis
gradients recomputed point by point, grid-point motion, charge motion).
Reference pieces: becke.cpp:79-176 (weights), gto.cpp:41-94 (basis and its
derivative), nnuclear.py:15-37 (potential), nwavefunction.cpp:161-197
(quadrature).
"""
from ctypes import byref, c_double, c_void_p

import numpy as np

from . import cext
from .cext import NapmoError, checked
from .fock import FockBuilder, _stream, _torch
from .grids import BeckeGrid
from .system import MolecularSystem


class GridChargeEnergy(object):
    """E(D, R) of species `species` on its own Becke grid (nrad x nang per
    centre) in the potential of the classical nuclei.

    Args:
        symbols: element symbols of the atoms, in order.
        species: 'e-' or a quantum nucleus species ('H_1' for quantum H).
        basis: electronic basis name.
        quantum: indices of atoms whose nuclei are a quantum species (5s5p).
    """

    def __init__(self, symbols, species='e-', basis='CC-PVDZ', quantum=(), nrad=75, nang=194,
                 reuse=True, precision='fp64'):
        self.symbols = list(symbols)
        self.species = species
        self.basis_name = basis
        self.quantum = tuple(quantum)
        self.nrad, self.nang = int(nrad), int(nang)
        # reuse: one grid, basis and plan, moved from geometry to geometry
        # (napmo_grid_set_centers, napmo_basis_set_origins,
        # napmo_fock_plan_refresh) instead of new objects per geometry
        self.reuse = bool(reuse)
        self._live = None
        # precision of the quadrature matrix V = dE/dD ('fp64' or 'int8x4');
        # the gradient kernel is FP64 in both
        self.precision = precision

    def system(self, R):
        """MolecularSystem at positions R (natom x 3, bohr), with the atom
        index of every centre of `species` and of every classical charge."""
        R = np.asarray(R, dtype=np.float64).reshape(-1, 3)
        ms = MolecularSystem()
        centres, charges = [], []
        for i, (sym, xyz) in enumerate(zip(self.symbols, R)):
            q = i in self.quantum
            ms.add_atom(sym, xyz, units='BOHR', basis_name=self.basis_name, quantum=q)
            if self.species == 'e-' or (q and self.species == sym + '_1'):
                centres.append(i)
            if not q:
                charges.append(i)
        if self.species not in ms:
            raise NapmoError('species %s not in the system' % self.species)
        return ms, centres, charges

    def _setup(self, R):
        ms, centres, charges = self.system(R)
        sp = ms[self.species]
        grid = BeckeGrid(sp, self.nrad, self.nang)
        qs = float(sp['charge'])
        Zq = np.array([[*ms.point_charges[k]['origin'], qs * ms.point_charges[k]['atomic_number']]
                       for k in range(len(charges))], dtype=np.float64).reshape(-1, 4)
        return ms, sp, grid, centres, charges, Zq

    def _objects(self, R):
        """(grid, basis, plan, centres, charges, Zq) at positions R."""
        R = np.asarray(R, dtype=np.float64).reshape(-1, 3)
        live = self._live
        if live is None:
            ms, sp, grid, centres, charges, Zq = self._setup(R)
            fb = FockBuilder(grid, sp['basis'], -1, precision=self.precision)
            obj = dict(ms=ms, grid=grid, basis=sp['basis'], fb=fb, centres=centres,
                       charges=charges, Zq=Zq, R=R.copy())
            if self.reuse:
                # atom of every basis function: the centre its origin sits on
                org = sp['basis'].origins()
                cen = R[centres]
                obj['func_centre'] = np.array(
                    [int(np.flatnonzero((cen == o).all(axis=1))[0]) for o in org])
                obj['qcharge'] = Zq[:, 3].copy()
                self._live = obj
            return obj
        if not np.array_equal(live['R'], R):
            cen = R[live['centres']]
            live['grid'].set_centers(cen)
            live['basis'].set_origins(cen[live['func_centre']])
            live['fb'].refresh()
            live['Zq'] = np.concatenate([R[live['charges']], live['qcharge'][:, None]], axis=1)
            live['R'] = R.copy()
        return live

    def quadrature_matrix(self, R):
        """(V, state): V = dE/dD on the device; state keeps the grid for the
        gradient."""
        torch = _torch()
        obj = self._objects(R)
        grid, fb, centres, charges, Zq = (obj['grid'], obj['fb'], obj['centres'],
                                          obj['charges'], obj['Zq'])
        x, y, z, _, _ = grid.device_arrays()
        v = torch.empty(grid.size, dtype=torch.float64, device='cuda')
        checked(cext.lib.napmo_gpu_nuclear_potential(
            grid.size, x, y, z, Zq.shape[0], np.ascontiguousarray(Zq), v.data_ptr(),
            torch.cuda.current_stream().cuda_stream))
        V = fb.quadrature(1.0, v)
        return V, dict(grid=grid, basis=obj['basis'], centres=centres, charges=charges, Zq=Zq,
                       natom=len(self.symbols), fb=fb, R=obj['R'].copy())

    def gradient(self, state, D):
        """(E, dE/dR [natom][3]) from the gradient kernel."""
        torch = _torch()
        if self.reuse:  # the shared objects may have moved since the forward
            self._objects(state['R'])
        D = torch.as_tensor(D, dtype=torch.float64, device='cuda').contiguous()
        nc = len(state['centres'])
        Zq = state['Zq']
        E = c_double()
        g = np.zeros((nc, 3))
        gq = np.zeros((max(1, Zq.shape[0]), 3))
        checked(cext.lib.napmo_grid_energy_gradient(
            state['grid']._this, state['basis']._this, D.data_ptr(), Zq.shape[0],
            np.ascontiguousarray(Zq).ctypes.data if Zq.shape[0] else None, byref(E),
            g.ctypes.data, gq.ctypes.data, _stream(torch, None)))
        out = np.zeros((state['natom'], 3))
        for k, a in enumerate(state['centres']):
            out[a] += g[k]
        for k, a in enumerate(state['charges']):
            out[a] += gq[k]
        return E.value, out

    def __call__(self, D, R):
        """E as a torch scalar differentiable in D (n x n) and R (natom x 3)."""
        return GridEnergyFunction.apply(D, R, self)


def _grid_energy_function():
    torch = _torch()

    class _Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, D, R, model):
            V, state = model.quadrature_matrix(R.detach().cpu().numpy())
            Dd = D.detach().to(device='cuda', dtype=torch.float64)
            E = (Dd * V).sum()
            ctx.model, ctx.state = model, state
            ctx.save_for_backward(D, R, V)
            return E.to(D.device)

        @staticmethod
        def backward(ctx, gE):
            D, R, V = ctx.saved_tensors
            gD = gR = None
            if ctx.needs_input_grad[0]:
                gD = (gE.to(V.device) * V).to(D.device)
            if ctx.needs_input_grad[1]:
                _, g = ctx.model.gradient(ctx.state, D.detach())
                gR = gE.to(R.device) * torch.as_tensor(g, dtype=R.dtype, device=R.device)
            return gD, gR, None

    return _Fn


class _Lazy(object):
    fn = None


class GridEnergyFunction(object):
    """torch.autograd.Function for E(D, R); see GridChargeEnergy."""

    @staticmethod
    def apply(D, R, model):
        if _Lazy.fn is None:
            _Lazy.fn = _grid_energy_function()
        return _Lazy.fn.apply(D, R, model)
