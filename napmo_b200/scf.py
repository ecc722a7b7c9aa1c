"""Grid-based closed-shell SCF of the electrons on the device.

The SCF loop of nAPMO's drivers (scf.py:80-144 single, 275-338 nsingle;
convergence.py:35-65; wavefunction.cpp:64-116) on top of the grid Fock build:

  H = T + V_ne: T and S analytic (napmo_basis_one_body; nAPMO takes them from
      libint), V_ne = phi diag(wb w v_ne) phi^T on the grid (nnuclear.py:15-37)
  per iteration, on the device:
      rho = diag(phi^T D phi), v_H = Poisson(rho)      (the hot path)
      J = phi diag(wb w v_H) phi^T
      exchange 'hf':    K_mu,nu = sum_i sum_p W phi_mu psi_i V[psi_i phi_nu]
                        (orbital-pair Poisson solves, as psi_numeric.py:186-215
                        does in the orbital basis; small systems)
               'lda-x': Slater exchange v_x = -(3 rho / pi)^(1/3) folded into
                        the quadrature (any size)
               'lda':   Slater exchange + VWN5 correlation (nAPMO's
                        Functional 'lda', napmo_gpu_lda_xc)
               'none':  Hartree
      F = H + J - K (or H + J + V_x), Pulay DIIS on FDS - SDF (6 vectors),
      F C = S C e by the generalised eigensolver, D = 2 C_occ C_occ^T.

The contractions rho and F run in the plan's precision ('fp64' or 'int8x4');
Poisson, DIIS and the diagonalisation are FP64 in both.
"""
import time

import numpy as np

from . import cext
from .cext import checked
from .fock import FockBuilder, _torch
from .grids import BeckeGrid, lebedev_get_order

CX = -(3.0 / np.pi) ** (1.0 / 3.0)          # Slater: v_x = CX rho^(1/3)
EX = 0.75 * CX                              # e_x = EX rho^(4/3)
PROTON_MASS = 1836.15267247                 # electron masses (napmo/data/constants.py)


def lda_xc(torch, rho):
    """(v_xc, e_xc per particle) of LDA exchange + VWN5 correlation of rho
    (device tensor), by napmo_gpu_lda_xc."""
    n = rho.numel()
    out = [torch.empty(n, dtype=torch.float64, device='cuda') for _ in range(4)]
    checked(cext.lib.napmo_gpu_lda_xc(n, rho.data_ptr(), *[o.data_ptr() for o in out],
                                      torch.cuda.current_stream().cuda_stream))
    xzk, xv, czk, cv = out
    return xv + cv, xzk + czk


def lda_xc_polarized(torch, rho_a, rho_b):
    """(v_xc of alpha, v_xc of beta, e_xc per particle of the total density)
    of spin-polarised LDA exchange + VWN5 correlation (device tensors), by
    napmo_gpu_lda_xc_polarized."""
    n = rho_a.numel()
    out = [torch.empty(n, dtype=torch.float64, device='cuda') for _ in range(6)]
    checked(cext.lib.napmo_gpu_lda_xc_polarized(n, rho_a.data_ptr(), rho_b.data_ptr(),
                                                *[o.data_ptr() for o in out],
                                                torch.cuda.current_stream().cuda_stream))
    xzk, xva, xvb, czk, cva, cvb = out
    return xva + cva, xvb + cvb, xzk + czk


def epc17_2_device(torch, rho_e, rho_n):
    """(energy per electron, v_e, v_n) of epc17-2 (device tensors)."""
    n = rho_e.numel()
    out = [torch.empty(n, dtype=torch.float64, device='cuda') for _ in range(3)]
    checked(cext.lib.napmo_gpu_epc17_2(n, rho_e.data_ptr(), rho_n.data_ptr(),
                                       *[o.data_ptr() for o in out],
                                       torch.cuda.current_stream().cuda_stream))
    return tuple(out)


def grid_exchange(torch, fb, phi, psi, W, max_bytes=1 << 31):
    """K_mu,nu = sum_i sum_p W phi_mu psi_i V[psi_i phi_nu], symmetrised (grid
    exchange of the orbitals psi, nocc x N, in the basis phi, n x N).  The
    pair densities psi_i phi_nu of as many orbitals as fit in max_bytes (with
    their potentials and weighted products) are solved in one library call.
    Their part of K is phi B^T with B_nu(p) = sum_i W psi_i(p) V[psi_i phi_nu](p):
    one pass over the potentials and one product over the grid (k products of
    n x n over N points each would run as skinny GEMMs far below the memory
    rate).  Returns (K, solves)."""
    n, N = phi.shape
    nocc = psi.shape[0]
    step = max(1, min(nocc, max_bytes // (3 * n * N * 8)))
    B = torch.zeros((n, N), dtype=torch.float64, device='cuda')
    for i0 in range(0, nocc, step):
        ps = psi[i0:i0 + step]
        k = ps.shape[0]
        V = fb.coulomb_potentials((ps[:, None, :] * phi[None, :, :]).reshape(k * n, N))
        B += (V.reshape(k, n, N) * (W * ps)[:, None, :]).sum(0)
    K = phi @ B.T
    return 0.5 * (K + K.T), nocc * n


def nuclear_repulsion(point_charges):
    E = 0.0
    for i, a in enumerate(point_charges):
        for b in point_charges[:i]:
            d = np.linalg.norm(np.asarray(a['origin']) - np.asarray(b['origin']))
            E += a['atomic_number'] * b['atomic_number'] / d
    return E


class GridRHF(object):
    """Closed-shell SCF of the electrons of a MolecularSystem on its Becke grid.

    Args:
        ms: MolecularSystem (all nuclei classical).
        nrad, nang: grid per atom (lists allowed).
        exchange: 'hf', 'lda-x', 'lda' (exchange + VWN5 correlation) or 'none'.
        precision: 'fp64' or 'int8x4' for rho and the quadratures.
        diis: number of DIIS vectors.
        hcore: 'grid' (V_ne by grid quadrature, as nnuclear.py) or 'analytic'
            (V_ne by the device one-electron integrals, as libint gives it to
            nAPMO's analytic wave function).
    """

    def __init__(self, ms, nrad=50, nang=110, lmax=None, exchange='hf', precision='fp64',
                 diis=6, hcore='grid'):
        torch = _torch()
        self.torch = torch
        e = ms['e-']
        self.ms = ms
        self.grid = BeckeGrid(e, nrad, nang)
        if lmax is None:
            lmax = 'per-atom' if isinstance(nang, (list, tuple)) else lebedev_get_order(nang) // 2
        self.fb = FockBuilder(self.grid, e['basis'], lmax)
        n, N = self.fb.n, self.grid.size
        self.n, self.N = n, N
        self.nocc = int(e['occupation'])
        S = np.zeros((n, n))
        T = np.zeros((n, n))
        checked(cext.lib.napmo_basis_one_body(e['basis']._this, S, T))
        dev = dict(device='cuda', dtype=torch.float64)
        self.S = torch.as_tensor(S, **dev)
        self.T = torch.as_tensor(T, **dev)
        q = np.array([[*pc['origin'], pc['atomic_number']] for pc in ms.point_charges],
                     dtype=np.float64).reshape(-1, 4)
        x, y, z, _, _ = self.grid.device_arrays()
        vne = torch.empty(N, **dev)
        checked(cext.lib.napmo_gpu_nuclear_potential(N, x, y, z, q.shape[0],
                                                     np.ascontiguousarray(q), vne.data_ptr(),
                                                     torch.cuda.current_stream().cuda_stream))
        if hcore == 'analytic':
            # device McMurchie-Davidson integrals (libint's role in nAPMO)
            self.V = torch.empty((n, n), **dev)
            checked(cext.lib.napmo_gpu_one_body(e['basis']._this, q.shape[0],
                                                np.ascontiguousarray(q).ctypes.data, None, None,
                                                self.V.data_ptr(),
                                                torch.cuda.current_stream().cuda_stream))
        elif hcore == 'grid':
            self.V = self.fb.quadrature(-1.0, vne)      # FP64: built before any precision switch
        else:
            raise ValueError("hcore must be 'grid' or 'analytic'")
        self.H = self.T + self.V
        self.Enn = nuclear_repulsion(ms.point_charges)
        self.W = torch.as_tensor(self.grid.becke_weights * self.grid.weights, **dev)
        self.exchange = exchange
        self.ndiis = int(diis)
        self.precision = precision
        self.fb.set_precision(precision)
        s, U = torch.linalg.eigh(self.S)
        self.X = U @ torch.diag(s.rsqrt()) @ U.T          # S^-1/2
        self.fock_builds = 0
        self.poisson_solves = 0

    # ------------------------------------------------------------ pieces
    def _phi(self):
        return self.fb.phi()[:, :self.N]

    def exchange_matrix(self, Cocc):
        """K_mu,nu = sum_i sum_p W phi_mu psi_i V[psi_i phi_nu] (symmetrised)."""
        phi = self._phi()
        K, solves = grid_exchange(self.torch, self.fb, phi, Cocc.T @ phi, self.W)
        self.poisson_solves += solves
        return K

    def fock(self, D, Cocc):
        """(F, E_electronic) for density D."""
        t = self.torch
        rho = self.fb.density(D)
        vH = self.fb.coulomb_potential(rho)
        self.fock_builds += 1
        self.poisson_solves += 1
        if self.exchange == 'lda':
            vxc, exc = lda_xc(t, rho)
            G = self.fb.quadrature(1.0, vH, vext=vxc)
            EJ = 0.5 * float((self.W * rho * vH).sum())
            Exc = float((self.W * rho * exc).sum())
            return self.H + G, float((D * self.H).sum()) + EJ + Exc
        if self.exchange == 'lda-x':
            r13 = t.clamp(rho, min=0.0) ** (1.0 / 3.0)
            G = self.fb.quadrature(1.0, vH, vext=CX * r13)
            EJ = 0.5 * float((self.W * rho * vH).sum())
            Ex = float((self.W * EX * rho * r13).sum())
            F = self.H + G
            return F, float((D * self.H).sum()) + EJ + Ex
        J = self.fb.quadrature(1.0, vH)
        F = self.H + J
        if self.exchange == 'hf':
            F = F - self.exchange_matrix(Cocc)
        return F, 0.5 * float((D * (self.H + F)).sum())

    def _diag(self, F):
        Fp = self.X.T @ F @ self.X
        e, Cp = self.torch.linalg.eigh(Fp)
        return e, self.X @ Cp

    # -------------------------------------------------------------- loop
    def run(self, maxiter=100, tol=1e-8, verbose=False):
        t = self.torch
        torch = t
        t0 = time.perf_counter()
        self.O, C = self._diag(self.H)                     # core guess
        Cocc = C[:, :self.nocc]
        D = 2.0 * Cocc @ Cocc.T
        Fs, errs, history = [], [], []
        E_prev = None
        converged = False
        for it in range(1, maxiter + 1):
            F, Eel = self.fock(D, Cocc)
            E = Eel + self.Enn
            err = F @ D @ self.S - self.S @ D @ F
            err = self.X.T @ err @ self.X
            Fs.append(F)
            errs.append(err)
            if len(Fs) > self.ndiis:
                Fs.pop(0)
                errs.pop(0)
            emax = float(err.abs().max())
            history.append((E, emax))
            if verbose:
                print('%3d %.12f %.3e' % (it, E, emax))
            if E_prev is not None and abs(E - E_prev) < tol and emax < 1e-4:
                converged = True
                break
            E_prev = E
            if len(Fs) > 1:
                F = _diis_extrapolate(torch, Fs, errs)
            e, C = self._diag(F)
            Cocc = C[:, :self.nocc]
            D = 2.0 * Cocc @ Cocc.T
            self.O = e
        torch.cuda.synchronize()
        self.D, self.C = D, C
        nel = float((D * self.S).sum())
        return dict(energy=E, iterations=it, converged=converged, seconds=time.perf_counter() - t0,
                    fock_builds=self.fock_builds, poisson_solves=self.poisson_solves,
                    electrons=nel, history=history)


def _diis_coefficients(torch, errs):
    """DIIS coefficients (summing to 1) of the stored iterations whose error
    combination has the least norm; errs[a] is iteration a's error matrix or a
    tuple of them (one per species, one DIIS over all).  The errors' overlap
    matrix is one product of their stacked, concatenated vectors."""
    ev = torch.stack([torch.cat([x.reshape(-1) for x in (e if isinstance(e, (tuple, list))
                                                          else (e,))]) for e in errs])
    m = ev.shape[0]
    B = torch.zeros((m + 1, m + 1), dtype=torch.float64, device='cuda')
    B[:m, :m] = ev @ ev.T
    B[m, :m] = -1.0
    B[:m, m] = -1.0
    rhs = torch.zeros(m + 1, dtype=torch.float64, device='cuda')
    rhs[m] = -1.0
    return torch.linalg.solve(B, rhs)[:m]


def _diis_extrapolate(torch, Fs, errs):
    """The DIIS combination of the stored Fock matrices."""
    return torch.tensordot(_diis_coefficients(torch, errs), torch.stack(Fs), dims=1)


class _Species(object):
    """One species on the shared grid: its Fock plan, S, H = T / mass +
    q V_nuc (classical charges), S^-1/2, occupation and DIIS history."""

    def __init__(self, grid, sp, point_charges, lmax, mass, precision, ndiis, torch):
        self.torch = torch
        self.fb = FockBuilder(grid, sp['basis'], lmax)
        n, N = self.fb.n, grid.size
        self.n, self.N = n, N
        self.q = float(sp['charge'])
        self.eta = float(sp['eta'])
        self.nocc = int(sp['occupation'])
        S = np.zeros((n, n))
        T = np.zeros((n, n))
        checked(cext.lib.napmo_basis_one_body(sp['basis']._this, S, T))
        dev = dict(device='cuda', dtype=torch.float64)
        self.S = torch.as_tensor(S, **dev)
        H = torch.as_tensor(T, **dev) / mass
        if point_charges:
            qc = np.array([[*pc['origin'], pc['atomic_number']] for pc in point_charges],
                          dtype=np.float64).reshape(-1, 4)
            x, y, z, _, _ = grid.device_arrays()
            vn = torch.empty(N, **dev)
            checked(cext.lib.napmo_gpu_nuclear_potential(
                N, x, y, z, qc.shape[0], np.ascontiguousarray(qc), vn.data_ptr(),
                torch.cuda.current_stream().cuda_stream))
            H = H + self.fb.quadrature(self.q, vn)      # FP64, before any precision switch
        self.H = H
        self.fb.set_precision(precision)
        s, U = torch.linalg.eigh(self.S)
        self.X = U @ torch.diag(s.rsqrt()) @ U.T
        self.ndiis = ndiis
        self.Fs, self.errs = [], []

    def diag(self, F):
        e, Cp = self.torch.linalg.eigh(self.X.T @ F @ self.X)
        C = self.X @ Cp
        Cocc = C[:, :self.nocc]
        return C, Cocc, self.eta * Cocc @ Cocc.T

    def diis(self, F, D):
        err = self.X.T @ (F @ D @ self.S - self.S @ D @ F) @ self.X
        self.Fs.append(F)
        self.errs.append(err)
        if len(self.Fs) > self.ndiis:
            self.Fs.pop(0)
            self.errs.pop(0)
        Fx = _diis_extrapolate(self.torch, self.Fs, self.errs) if len(self.Fs) > 1 else F
        return Fx, float(err.abs().max())


class GridAPMO(object):
    """APMO closed-shell SCF of the electrons and one quantum-nucleus species
    (nAPMO's multi-species drivers, scf.py:146-273 / psi_hybrid.py:81-110):
    both species on one Becke grid over all atoms; the electron-nucleus
    coupling is the grid Coulomb quadrature of the other species' density
    (potential from the device Poisson solve); electron exchange from
    orbital-pair Poisson solves; a single quantum nucleus has no self
    interaction (J - K = 0); classical nuclei enter H of both species.

    E = sum_s tr(D_s H_s) + 1/2 tr(D_e (J_e - K_e))
        + 1/2 q_e q_n (<rho_e|V[rho_n]> + <rho_n|V[rho_e]>) + E_nn(classical)
    (the coupling as nAPMO's 1/2 sum_s tr(D_s J_s), scf.py:494-520)

    exchange='lda' replaces the electrons' HF exchange by LDA exchange +
    VWN5 correlation (nAPMO's Functional 'lda'); correlation='epc17-2' adds
    the electron-proton correlation functional of the two densities.
    """

    def __init__(self, ms, nuclear='H_1', nrad=100, nang=302, lmax=None, precision='fp64',
                 diis=6, mass=PROTON_MASS, exchange='hf', correlation=None):
        torch = _torch()
        self.torch = torch
        if exchange not in ('hf', 'lda'):
            raise ValueError("exchange must be 'hf' or 'lda'")
        if correlation not in (None, 'epc17-2'):
            raise NotImplementedError(str(correlation) + ' Functional NOT available!')
        self.exchange = exchange            # electrons: HF exchange or LDA (x + VWN5 c)
        self.correlation = correlation      # electron-nucleus: None or epc17-2
        self.ms = ms
        self.grid = BeckeGrid(ms['e-'], nrad, nang)
        if lmax is None:
            lmax = 'per-atom' if isinstance(nang, (list, tuple)) else lebedev_get_order(nang) // 2
        self.W = torch.as_tensor(self.grid.becke_weights * self.grid.weights, device='cuda',
                                 dtype=torch.float64)
        self.e = _Species(self.grid, ms['e-'], ms.point_charges, lmax, 1.0, precision, diis,
                          torch)
        self.nuc = _Species(self.grid, ms[nuclear], ms.point_charges, lmax, mass, precision,
                            diis, torch)
        if self.nuc.nocc != 1:
            raise ValueError('one quantum nucleus of the species is supported')
        self.Enn = nuclear_repulsion(ms.point_charges)
        self._nuclear = nuclear
        self.poisson_solves = 0

    def _exchange(self, Cocc):
        sp = self.e
        phi = sp.fb.phi()[:, :sp.N]
        K, solves = grid_exchange(self.torch, sp.fb, phi, Cocc.T @ phi, self.W)
        self.poisson_solves += solves
        return K

    def fock(self, De, Dn, Ce=None):
        """(F_e, F_n, E) for densities De, Dn (Ce: electron orbitals, for HF
        exchange).  Both species share the grid, so the electron-nucleus
        functional (epc17-2, interspecies_correlation.py:36-68) is evaluated
        point by point and its energy sum_p W rho_e e_epc enters once, its
        potentials the Fock matrices of both species (psi_analytic.py:219-258)."""
        e, n, t = self.e, self.nuc, self.torch
        qq = e.q * n.q
        rho_e = e.fb.density(De)
        rho_n = n.fb.density(Dn)
        v_e = e.fb.coulomb_potential(rho_e)
        v_n = e.fb.coulomb_potential(rho_n)
        self.poisson_solves += 2
        ext_e, ext_n, E_xc = qq * v_n, None, 0.0
        if self.exchange == 'lda':
            vxc, exc = lda_xc(t, rho_e)
            ext_e = ext_e + vxc
            E_xc += float((self.W * rho_e * exc).sum())
        if self.correlation == 'epc17-2':
            ene, pe, pn = epc17_2_device(t, rho_e, rho_n)
            ext_e = ext_e + pe
            ext_n = pn
            E_xc += float((self.W * rho_e * ene).sum())
        # electrons: q_e^2 J_e + q_e q_n J[rho_n] (+ v_xc, epc) - K_e;
        # nucleus: q_n q_e J[rho_e] (+ epc)
        Fe = e.H + e.fb.quadrature(e.q * e.q, v_e, vext=ext_e)
        E_K = 0.0
        if self.exchange == 'hf':
            K = self._exchange(Ce[:, :e.nocc])
            Fe = Fe - K
            E_K = -0.5 * float((De * K).sum())
        Fn = n.H + n.fb.quadrature(qq, v_e, vext=ext_n)
        # nAPMO's coupling energy: 1/2 sum_s tr(D_s J_s) (scf.py:494-520), the
        # mean of <rho_e|V[rho_n]> and <rho_n|V[rho_e]> (equal up to the grid)
        coup = 0.5 * qq * (float((self.W * rho_e * v_n).sum()) +
                           float((self.W * rho_n * v_e).sum()))
        E_J = 0.5 * e.q * e.q * float((self.W * rho_e * v_e).sum())
        E = (float((De * e.H).sum()) + E_J + E_K + E_xc + float((Dn * n.H).sum()) + coup +
             self.Enn)
        return Fe, Fn, E

    def run(self, maxiter=100, tol=1e-8, verbose=False):
        """SCF from a guess with the quantum nuclei as point charges (electrons)
        and the nucleus in that electron density's field; one DIIS over both
        species (concatenated error vectors, shared coefficients)."""
        torch = self.torch
        e, n = self.e, self.nuc
        t0 = time.perf_counter()
        qq = e.q * n.q
        # guess: electrons with the quantum nuclei as classical charges
        qpos = np.array([[*p['origin'], 1.0] for p in self.ms[self._nuclear]['particles']],
                        dtype=np.float64).reshape(-1, 4)
        x, y, z, _, _ = self.grid.device_arrays()
        vq = torch.empty(self.grid.size, device='cuda', dtype=torch.float64)
        checked(cext.lib.napmo_gpu_nuclear_potential(
            self.grid.size, x, y, z, qpos.shape[0], np.ascontiguousarray(qpos), vq.data_ptr(),
            torch.cuda.current_stream().cuda_stream))
        prec = e.fb.precision
        e.fb.set_precision('fp64')
        Hg = e.H + e.fb.quadrature(e.q * n.q, vq)
        e.fb.set_precision(prec)
        Ce, _, De = e.diag(Hg)
        v_e = e.fb.coulomb_potential(e.fb.density(De))
        Cn, _, Dn = n.diag(n.H + n.fb.quadrature(qq, v_e))
        self.poisson_solves += 1
        Fs, errs = [], []
        E_prev, history, converged = None, [], False
        for it in range(1, maxiter + 1):
            Fe, Fn, E = self.fock(De, Dn, Ce)
            err_e = e.X.T @ (Fe @ De @ e.S - e.S @ De @ Fe) @ e.X
            err_n = n.X.T @ (Fn @ Dn @ n.S - n.S @ Dn @ Fn) @ n.X
            Fs.append((Fe, Fn))
            errs.append((err_e, err_n))
            if len(Fs) > e.ndiis:
                Fs.pop(0)
                errs.pop(0)
            emax = (float(err_e.abs().max()), float(err_n.abs().max()))
            history.append((E,) + emax)
            if verbose:
                print('%3d %.12f %.2e %.2e' % ((it, E) + emax))
            if E_prev is not None and abs(E - E_prev) < tol and max(emax) < 1e-4:
                converged = True
                break
            E_prev = E
            m = len(Fs)
            if m > 1:
                c = _diis_coefficients(torch, errs)
                Fe = torch.tensordot(c, torch.stack([f[0] for f in Fs]), dims=1)
                Fn = torch.tensordot(c, torch.stack([f[1] for f in Fs]), dims=1)
            Ce, _, De = e.diag(Fe)
            Cn, _, Dn = n.diag(Fn)
        torch.cuda.synchronize()
        return dict(energy=E, iterations=it, converged=converged,
                    seconds=time.perf_counter() - t0, poisson_solves=self.poisson_solves,
                    electrons=float((De * e.S).sum()), nuclei=float((Dn * n.S).sum()),
                    history=history)


def spin_occupations(nelectron, multiplicity=None):
    """(n_alpha, n_beta) of `nelectron` electrons at a spin multiplicity, as
    nAPMO splits the species e- into e-alpha and e-beta
    (molecular_system.py:214-290): the default multiplicity is 1 for an even
    and 2 for an odd count; the unpaired electrons are alpha."""
    if not multiplicity:
        multiplicity = (nelectron % 2) + 1
    unpaired = multiplicity - 1
    left = nelectron - unpaired
    if left < 0 or left % 2 != 0:
        raise ValueError('Bad charge / multiplicity')
    return left // 2 + unpaired, left // 2


class GridMultiSCF(object):
    """Unrestricted SCF of several species on one Becke grid: the electrons
    as the two spin species e-alpha and e-beta (eta = 1 each, as nAPMO splits
    them for method 'uhf', molecular_system.py:214-290), optionally with one
    quantum-nucleus species (APMO-UHF).  Every species sees the Coulomb
    potential of every other (q_s q_t J[rho_t], grid quadrature of the device
    Poisson potentials) and of the classical nuclei; each spin species has
    its own HF exchange from its occupied orbitals (orbital-pair Poisson
    solves); a single quantum nucleus has no self-interaction.

    E = sum_s tr(D_s H_s) + 1/2 sum_{s,t} q_s q_t <rho_s|V[rho_t]>
        - 1/2 sum_{s in e} tr(D_s K_s) + E_nn(classical)
    (self terms s = t only for the electron species).

    Args:
        ms: MolecularSystem (quantum nuclei as their own species).
        nuclear: symbol of the quantum-nucleus species or None.
        charge: molecular charge (electrons = sum Z - charge).
        multiplicity: spin multiplicity (default 1 or 2 by parity).
        exchange: 'hf', 'lda' (spin-polarised LDA exchange + VWN5 correlation
            of the two spin densities, nAPMO's DFT for open shells) or 'none'
            for the electrons.
    """

    def __init__(self, ms, nuclear=None, nrad=50, nang=110, lmax=None, charge=0,
                 multiplicity=None, precision='fp64', diis=6, mass=PROTON_MASS, exchange='hf'):
        torch = _torch()
        self.torch = torch
        if exchange not in ('hf', 'lda', 'none'):
            raise ValueError("exchange must be 'hf', 'lda' or 'none' in the unrestricted drivers")
        self.exchange = exchange
        self.ms = ms
        e = ms['e-']
        self.grid = BeckeGrid(e, nrad, nang)
        if lmax is None:
            lmax = 'per-atom' if isinstance(nang, (list, tuple)) else lebedev_get_order(nang) // 2
        self.W = torch.as_tensor(self.grid.becke_weights * self.grid.weights, device='cuda',
                                 dtype=torch.float64)
        nel = int(round(e['size'])) - int(charge)
        self.nalpha, self.nbeta = spin_occupations(nel, multiplicity)
        self.species = []
        for occ in (self.nalpha, self.nbeta):
            sp = dict(e, eta=1.0, occupation=occ)
            self.species.append(_Species(self.grid, sp, ms.point_charges, lmax, 1.0, precision,
                                         diis, torch))
        self.is_electron = [True, True]
        self._nuclear = nuclear
        if nuclear is not None:
            self.species.append(_Species(self.grid, ms[nuclear], ms.point_charges, lmax, mass,
                                         precision, diis, torch))
            self.is_electron.append(False)
            if self.species[-1].nocc != 1:
                raise ValueError('one quantum nucleus of the species is supported')
        self.ndiis = int(diis)
        self.Enn = nuclear_repulsion(ms.point_charges)
        self.poisson_solves = 0

    def _exchange(self, sp, Cocc):
        phi = sp.fb.phi()[:, :sp.N]
        K, solves = grid_exchange(self.torch, sp.fb, phi, Cocc.T @ phi, self.W)
        self.poisson_solves += solves
        return K

    def fock(self, Ds, Cs):
        """(list of F_s, E) for densities Ds and orbitals Cs."""
        sps = self.species
        rhos = [sp.fb.density(D) for sp, D in zip(sps, Ds)]
        vs = [sps[0].fb.coulomb_potential(r) for r in rhos]
        self.poisson_solves += len(rhos)
        Fs, E = [], self.Enn
        vxc = [None] * len(sps)
        if self.exchange == 'lda':
            va, vb, exc = lda_xc_polarized(self.torch, rhos[0], rhos[1])
            vxc[0], vxc[1] = va, vb
            E += float((self.W * (rhos[0] + rhos[1]) * exc).sum())
        for s, sp in enumerate(sps):
            pot = None
            for u, (tp, v) in enumerate(zip(sps, vs)):
                if u == s and not self.is_electron[s]:
                    continue
                term = (sp.q * tp.q) * v
                pot = term if pot is None else pot + term
            F = sp.H + sp.fb.quadrature(1.0, pot, vext=vxc[s])
            E += float((Ds[s] * sp.H).sum()) + 0.5 * float((self.W * rhos[s] * pot).sum())
            if self.exchange == 'hf' and self.is_electron[s] and sp.nocc > 0:
                K = self._exchange(sp, Cs[s][:, :sp.nocc])
                F = F - K
                E -= 0.5 * float((Ds[s] * K).sum())
            Fs.append(F)
        return Fs, E

    def guess(self):
        """Electrons from the core Hamiltonian with the quantum nuclei as unit
        point charges; the nucleus in that electron density's field."""
        torch = self.torch
        sps = self.species
        H = sps[0].H
        if self._nuclear is not None:
            qpos = np.array([[*p['origin'], 1.0] for p in self.ms[self._nuclear]['particles']],
                            dtype=np.float64).reshape(-1, 4)
            x, y, z, _, _ = self.grid.device_arrays()
            vq = torch.empty(self.grid.size, device='cuda', dtype=torch.float64)
            checked(cext.lib.napmo_gpu_nuclear_potential(
                self.grid.size, x, y, z, qpos.shape[0], np.ascontiguousarray(qpos),
                vq.data_ptr(), torch.cuda.current_stream().cuda_stream))
            prec = sps[0].fb.precision
            sps[0].fb.set_precision('fp64')
            H = H + sps[0].fb.quadrature(sps[0].q * sps[-1].q, vq)
            sps[0].fb.set_precision(prec)
        Cs, Ds = [], []
        for sp in sps[:2]:
            C, _, D = sp.diag(H)
            Cs.append(C)
            Ds.append(D)
        if self._nuclear is not None:
            nuc = sps[2]
            v_e = sps[0].fb.coulomb_potential(sps[0].fb.density(Ds[0] + Ds[1]))
            self.poisson_solves += 1
            C, _, D = nuc.diag(nuc.H + nuc.fb.quadrature(sps[0].q * nuc.q, v_e))
            Cs.append(C)
            Ds.append(D)
        return Cs, Ds

    def run(self, maxiter=100, tol=1e-8, verbose=False):
        """SCF from guess(); one DIIS over all species (concatenated error
        vectors, shared coefficients); stops at |dE| < tol with every
        max |X^T (FDS - SDF) X| < 1e-4."""
        torch = self.torch
        sps = self.species
        t0 = time.perf_counter()
        Cs, Ds = self.guess()
        Fh, errs = [], []
        E_prev, history, converged = None, [], False
        for it in range(1, maxiter + 1):
            Fs, E = self.fock(Ds, Cs)
            err = [sp.X.T @ (F @ D @ sp.S - sp.S @ D @ F) @ sp.X
                   for sp, F, D in zip(sps, Fs, Ds)]
            Fh.append(Fs)
            errs.append(err)
            if len(Fh) > self.ndiis:
                Fh.pop(0)
                errs.pop(0)
            emax = tuple(float(x.abs().max()) for x in err)
            history.append((E,) + emax)
            if verbose:
                print('%3d %.12f %s' % (it, E, ' '.join('%.2e' % x for x in emax)))
            if E_prev is not None and abs(E - E_prev) < tol and max(emax) < 1e-4:
                converged = True
                break
            E_prev = E
            m = len(Fh)
            if m > 1:
                c = _diis_coefficients(torch, errs)
                Fs = [torch.tensordot(c, torch.stack([f[s] for f in Fh]), dims=1)
                      for s in range(len(sps))]
            Cs, Ds = [], []
            for sp, F in zip(sps, Fs):
                C, _, D = sp.diag(F)
                Cs.append(C)
                Ds.append(D)
        torch.cuda.synchronize()
        out = dict(energy=E, iterations=it, converged=converged,
                   seconds=time.perf_counter() - t0, poisson_solves=self.poisson_solves,
                   alpha=float((Ds[0] * sps[0].S).sum()), beta=float((Ds[1] * sps[1].S).sum()),
                   history=history, D=[D for D in Ds])
        if self._nuclear is not None:
            out['nuclei'] = float((Ds[2] * sps[2].S).sum())
        return out


class GridUHF(GridMultiSCF):
    """Unrestricted grid SCF of the electrons (nAPMO's method 'uhf'):
    GridMultiSCF without quantum nuclei."""

    def __init__(self, ms, nrad=50, nang=110, **kw):
        super(GridUHF, self).__init__(ms, None, nrad, nang, **kw)
