"""Numerical-orbital Hartree-Fock on the grid, on the device.

nAPMO's numerical wave function (PSIN, napmo/wavefunction/psi_numeric.py:23-507)
holds each occupied orbital as its values on the molecular Becke grid; its
Becke-Dickson optimiser (PSIO_BECKE, napmo/wavefunction/psi_optimization.py:
124-221; A. D. Becke and R. M. Dickson, J. Chem. Phys. 92, 3610 (1990))
improves them from the residual R = (T + V - e) psi by one radial ODE per
atom and (l, m), then re-diagonalises the Fock operator in the space of the
orbitals and their corrections.

Device entry points (libnapmo):
  napmo_gpu_kinetic          compute_kinetic   (nkinetic.py:15-73)
  napmo_gpu_dpsi             compute_dpsi      (ndpsi.py:15-89)
  napmo_gpu_operator_matrix  get_operator_matrix (psi_numeric.py:406-424)
  napmo_gpu_poisson          compute_coulomb   (ntwobody.py:15-46)
The small matrix steps go through wavefunction_guess_hcore / wavefunction_iterate
(the libnapmo SCF step) as nAPMO calls them.  Orbitals, potentials and
operator images stay on the device as [k][npoint] tensors; torch holds them.
"""
import numpy as np

from . import cext
from .cext import checked
from .fock import _torch
from .grids import coulomb_potential_device, lebedev_get_order
from .wavefunction import WaveFunction


def INDEX(i, j):
    """Packed index of the pair (i, j) (psi_numeric.py:16-20)."""
    return i * (i + 1) // 2 + j if i > j else j * (j + 1) // 2 + i


class GridOperators(object):
    """The numerical-orbital operators of one BeckeGrid at expansion order lmax."""

    def __init__(self, grid, lmax=None):
        self.t = _torch()
        self.grid = grid
        self.N = grid.size
        self.lmax = int(lebedev_get_order(grid.nang) // 2 if lmax is None else lmax)

    def _stream(self):
        return self.t.cuda.current_stream().cuda_stream

    def rows(self, x):
        """x as contiguous FP64 device rows [k][npoint]."""
        t = self.t
        if not isinstance(x, t.Tensor):
            x = t.as_tensor(np.ascontiguousarray(x, dtype=np.float64))
        return x.to(device='cuda', dtype=t.float64).reshape(-1, self.N).contiguous()

    def kinetic(self, psi, scale=1.0):
        """scale * (-1/2 laplacian psi_k) for every row."""
        psi = self.rows(psi)
        out = self.t.empty_like(psi)
        checked(cext.lib.napmo_gpu_kinetic(self.grid._this, self.lmax, psi.shape[0],
                                           psi.data_ptr(), self.N, float(scale), out.data_ptr(),
                                           self._stream()))
        return out

    def dpsi(self, phi, resid, vtot, doi, oi, mass_inv):
        """Becke-Dickson corrections of the rows of phi."""
        phi, resid, vtot = self.rows(phi), self.rows(resid), self.rows(vtot)
        k = phi.shape[0]
        doi = np.ascontiguousarray(np.asarray(doi, dtype=np.float64).reshape(-1)[:k])
        oi = np.ascontiguousarray(np.asarray(oi, dtype=np.float64).reshape(-1)[:k])
        if resid.shape[0] != k or vtot.shape[0] != k or doi.size != k or oi.size != k:
            raise cext.NapmoError('phi, resid, vtot, doi and oi must hold the same orbitals')
        out = self.t.empty_like(phi)
        checked(cext.lib.napmo_gpu_dpsi(self.grid._this, self.lmax, k, phi.data_ptr(),
                                        resid.data_ptr(), vtot.data_ptr(), self.N, doi, oi,
                                        float(mass_inv), out.data_ptr(), self._stream()))
        return out

    def matrix(self, A, B):
        """M[i][j] = integral A_i B_j over the grid (Becke and quadrature weights)."""
        A, B = self.rows(A), self.rows(B)
        M = self.t.empty((A.shape[0], B.shape[0]), dtype=self.t.float64, device='cuda')
        checked(cext.lib.napmo_gpu_operator_matrix(self.grid._this, A.shape[0], B.shape[0],
                                                   A.data_ptr(), self.N, B.data_ptr(), self.N,
                                                   M.data_ptr(), self._stream()))
        return M

    def coulomb(self, rho):
        """V_H[rho] at the grid points."""
        rho = self.rows(rho).reshape(-1)
        v = self.t.empty(self.N, dtype=self.t.float64, device='cuda')
        coulomb_potential_device(self.grid, rho, self.lmax, v)
        return v

    def coulomb_many(self, rho):
        """V_H of every row of rho, in one library call."""
        rho = self.rows(rho)
        v = self.t.empty_like(rho)
        checked(cext.lib.napmo_gpu_poisson_many(self.grid._this, rho.shape[0], rho.data_ptr(),
                                                self.N, self.lmax, v.data_ptr(), self._stream()))
        return v


def _like_input(x, out):
    t = _torch()
    return out if isinstance(x, t.Tensor) else out.cpu().numpy()


def compute_kinetic(grid, psi, lmax):
    """-1/2 laplacian of psi at every grid point (nkinetic.py:15-73)."""
    ops = GridOperators(grid, lmax)
    return _like_input(psi, ops.kinetic(psi).reshape(-1))


def compute_dpsi(grid, lmax, phi, doi, oi, ri, V_tot, mass_inv):
    """Becke-Dickson correction of one orbital (ndpsi.py:15-89)."""
    ops = GridOperators(grid, lmax)
    return _like_input(phi, ops.dpsi(phi, ri, V_tot, [doi], [oi], mass_inv).reshape(-1))


class PSIN(object):
    """Numerical orbitals of one species (psi_numeric.py:23-175, 241-424).

    Args:
        grid: the species' BeckeGrid.
        gbasis: basis values on the grid [nbasis][npoint] (device or host).
        C: coefficients of the starting (basis-set) orbitals [nbasis][nbasis].
        O: their orbital energies (the first ndim start the optimiser).
        occupation: occupied orbitals; ndim defaults to it (1 when 0).
        point_charges: [(Z, (x, y, z))] in bohr; pce: their repulsion energy.
        eta, kappa, charge, mass: species constants (electrons 2, -1, -1, 1).
        size: number of particles (default eta x occupation).
    """

    def __init__(self, grid, gbasis, C, O, occupation, point_charges, pce=0.0, ndim=None,
                 lmax=None, eta=2.0, kappa=-1.0, charge=-1.0, mass=1.0, size=None):
        t = self.t = _torch()
        self.ops = GridOperators(grid, lmax)
        self.grid, self.N, self.lmax = grid, grid.size, self.ops.lmax
        self.occupation = int(occupation)
        self.ndim = int(ndim) if ndim else (self.occupation if self.occupation > 0 else 1)
        self.eta, self.kappa, self.x_factor = float(eta), float(kappa), float(kappa) / float(eta)
        self.charge, self.mass_inv, self.pce = float(charge), 1.0 / float(mass), float(pce)
        self.wf = WaveFunction(self.ndim, self.occupation, eta, kappa)
        self._prev_O = np.asarray(O, dtype=np.float64).copy()
        # point-charge potential sum_A Z_A / |r - R_A| (nnuclear.py:15-37)
        q = np.array([[*np.asarray(R, dtype=np.float64), Z] for Z, R in point_charges],
                     dtype=np.float64).reshape(-1, 4)
        x, y, z, _, _ = grid.device_arrays()
        self.Vnuc = t.empty(self.N, dtype=t.float64, device='cuda')
        checked(cext.lib.napmo_gpu_nuclear_potential(self.N, x, y, z, q.shape[0],
                                                     np.ascontiguousarray(q),
                                                     self.Vnuc.data_ptr(), self.ops._stream()))
        gb = self.ops.rows(gbasis)
        Cd = t.as_tensor(np.asarray(C, dtype=np.float64), device='cuda')
        self.psi = Cd.T @ gb                      # compute_psi_from_cm: row j = sum_k C[k,j] phi_k
        # two-body terms whenever the species has particles (psi_numeric.py:81-83)
        size = self.eta * self.occupation if size is None else size
        self.calculate_2body = size > 0
        self.Jpot = t.zeros(self.N, dtype=t.float64, device='cuda')
        self.Kpot = t.zeros((self.ndim, self.N), dtype=t.float64, device='cuda')
        self.initialize()
        self.optimizer = PSIO_BECKE(self)

    # ------------------------------------------------------ one-body part
    def initialize(self):
        self.normalize()
        self.compute_1body()
        self.compute_guess()

    def normalize(self):
        S = self.ops.matrix(self.psi[:self.ndim], self.psi[:self.ndim])
        self.psi = self.psi[:self.ndim] * S.diagonal().rsqrt()[:, None]
        self.S = self.ops.matrix(self.psi, self.psi)

    def compute_1body(self):
        self.Tgrid = self.ops.kinetic(self.psi, self.mass_inv)
        self.T = self.ops.matrix(self.psi, self.Tgrid)
        self.Vgrid = self.psi * self.Vnuc * self.charge
        self.V = self.ops.matrix(self.psi, self.Vgrid)
        self.H = self.T + self.V

    def _to_wf(self, **mats):
        for name, m in mats.items():
            getattr(self.wf, name)[:] = m.cpu().numpy() if hasattr(m, 'cpu') else m

    def compute_guess(self):
        self._to_wf(S=self.S, H=self.H)
        self.wf.guess_hcore()

    # ------------------------------------------------------ two-body part
    def compute_density(self):
        self.Dgrid = self.psi * self.psi * self.eta

    def compute_2body(self):
        """Coulomb and exchange potentials and G (psi_numeric.py:155-215)."""
        t = self.t
        n = self.ndim
        self.G = t.zeros((n, n), dtype=t.float64, device='cuda')
        if not self.calculate_2body:
            return
        self.compute_density()
        self.Jpot = self.ops.coulomb(self.Dgrid.sum(dim=0))
        G = self.ops.matrix(self.psi, self.psi * self.Jpot)
        if self.x_factor != 0.0:
            # K_j = sum_kl psi_k V[psi_l psi_j] D_kl = sum_l V[psi_l psi_j] chi_l with
            # chi_l = sum_k D_kl psi_k; each pair potential (INDEX packing, s >= v)
            # is used as soon as it is solved, so memory stays O(n N)
            D = t.as_tensor(self.wf.D.copy(), device='cuda')
            chi = D.T @ self.psi
            K = t.zeros((n, self.N), dtype=t.float64, device='cuda')
            for s in range(n):
                pots = self.ops.coulomb_many(self.psi[s] * self.psi[:s + 1])
                for v in range(s + 1):
                    K[v] += pots[v] * chi[s]
                    if s != v:
                        K[s] += pots[v] * chi[v]
            self.Kpot = K
            E = self.ops.matrix(self.psi, self.Kpot)
            E = t.triu(E) + t.triu(E, 1).T
            G = G + self.x_factor * E
        self.G = G * self.charge ** 2

    def build_fock(self):
        self.F = self.H + self.G

    def iterate(self):
        """F C = S C e, D = eta C_occ C_occ^T, energy (wavefunction.cpp:64-116)."""
        n = self.ndim
        self._to_wf(S=self.S, H=self.H, G=self.G, J=np.zeros((n, n)), F=self.F)
        self.wf.iterate()

    @property
    def O(self):
        return self.wf.O.copy()

    @property
    def energy(self):
        return self.wf.energy

    def get_operator_matrix(self, Operator):
        """M[i][j] = integral psi_i Operator_j over the grid, for the rows
        Operator_j = O psi_j (psi_numeric.py:406-424)."""
        return self.ops.matrix(self.psi, Operator)

    def compute_overlap(self):
        """S of the current orbitals (psi_numeric.py:125-133)."""
        self.S = self.ops.matrix(self.psi, self.psi)
        return self.S

    # ---------------------------------------------------------- optimiser
    def optimize_psi(self):
        self.psi = self.optimizer.optimize(self)[:self.ndim]
        self.normalize()
        self.compute_1body()


class PSIO_BECKE(object):
    """Becke-Dickson optimiser of a PSIN (psi_optimization.py:124-221): the
    orbitals and their corrections span a 2 ndim space in which the grid Fock
    operator is diagonalised."""

    def __init__(self, psin):
        self.ndim = 2 * psin.ndim
        self.wf = WaveFunction(self.ndim, psin.occupation, psin.eta, psin.kappa)
        self.prev_O = psin._prev_O.copy()
        self.delta_orb = np.zeros(self.ndim)
        self.delta_e = np.zeros(self.ndim)
        self.iterations = 1
        self.asymmetry = 0.0

    def optimize(self, psi):
        t = psi.t
        ops = psi.ops
        n = psi.ndim
        # potential acting on each orbital, residual, energy correction
        V_tot = psi.Vgrid + psi.psi * psi.Jpot + psi.Kpot * psi.x_factor
        prev = t.as_tensor(self.prev_O[:n], dtype=t.float64, device='cuda')
        R = psi.Tgrid + V_tot - prev[:, None] * psi.psi
        self.delta_e = ops.matrix(R, psi.psi).diagonal().cpu().numpy()
        self.delta_psi = ops.dpsi(psi.psi, R, V_tot, self.delta_e, self.prev_O[:n], psi.mass_inv)
        ext = t.cat([psi.psi, self.delta_psi])
        m = ext.shape[0]
        # Fock operator of the extended space (the density is the current one)
        S = ops.matrix(ext, ext)
        Hgrid = ops.kinetic(ext, psi.mass_inv) + ext * psi.Vnuc * psi.charge
        Fgrid = Hgrid
        if psi.calculate_2body:
            Jgrid = ext * psi.Jpot
            # K_v = sum_s ext_s V[ext_s ext_v], each pair potential solved once
            # and used at once (memory O(m N))
            Kgrid = t.zeros_like(ext)
            for s in range(m):
                pots = ops.coulomb_many(ext[s] * ext[:s + 1])
                for v in range(s + 1):
                    Kgrid[v] += ext[s] * pots[v]
                    if s != v:
                        Kgrid[s] += ext[v] * pots[v]
            Fgrid = Hgrid + Jgrid - Kgrid
        F = ops.matrix(ext, Fgrid)
        self.asymmetry = float((F - F.T).abs().max())
        F = (F + F.T) / 2.0
        self.S_ext, self.F_ext = S, F
        z = np.zeros((m, m))
        for name, val in (('S', S.cpu().numpy()), ('F', F.cpu().numpy()), ('H', z), ('G', z),
                          ('J', z)):
            getattr(self.wf, name)[:] = val
        self.wf.iterate()
        self.delta_orb = self.wf.O[:n] - psi.O
        self.prev_O = psi.O
        self.iterations += 1
        C = t.as_tensor(self.wf.C.copy(), device='cuda')
        return C.T @ ext


def optimize(psin, maxiter=100, tol=1e-8, verbose=False):
    """The Becke-Dickson SCF of nAPMO's numerical solver
    (test_psi_numeric_becke_*.py, hf_solver.py): one grid Fock step from the
    basis-set orbitals, then optimiser step + Fock step until the total energy
    changes by less than tol.  Returns a dict (energy, iterations, history)."""
    psin.compute_2body()
    psin.build_fock()
    psin.iterate()
    history = [psin.energy + psin.pce]
    E_prev = 0.0
    converged = False
    it = 0
    for it in range(1, maxiter + 1):
        psin.optimize_psi()
        psin.compute_2body()
        psin.build_fock()
        psin.iterate()
        E = psin.energy + psin.pce
        history.append(E)
        if verbose:
            print('%4d %.14f %.3e' % (it, E, abs(E - E_prev)))
        if abs(E - E_prev) < tol:
            converged = True
            break
        E_prev = E
    return dict(energy=history[-1], iterations=it, converged=converged, history=history)


def from_grid_rhf(rhf, grid=None, lmax=None):
    """A PSIN started from a converged GridRHF (its basis, orbitals and
    energies), on the RHF's own grid or another BeckeGrid of the electrons."""
    t = _torch()
    ms = rhf.ms
    e = ms['e-']
    if grid is None:
        grid, gb = rhf.grid, rhf.fb.phi()[:, :rhf.N]
    else:
        gb = t.as_tensor(np.ascontiguousarray(e['basis'].compute(grid.points).T), device='cuda')
    pcs = [(pc['atomic_number'], pc['origin']) for pc in ms.point_charges]
    from .scf import nuclear_repulsion
    return PSIN(grid, gb, rhf.C.cpu().numpy(), rhf.O.cpu().numpy(), int(e['occupation']), pcs,
                pce=nuclear_repulsion(ms.point_charges), lmax=lmax)
