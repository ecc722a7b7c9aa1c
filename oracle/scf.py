"""ORACLE -- test infrastructure only (the GPU tests, the fixture script
tests/golden/make_scf_golden.py and bench.py's reference leg use it as the
checker; the napmo_b200 package never imports it).

Host restatement of the grid SCF drivers, assembled from the oracle's pieces
of nAPMO's path:

  * grid: oracle.Grid (atomic_grid.cpp:12-51, becke.cpp:12-176);
  * basis on the grid: oracle.basis_compute (basis_set.cpp:69-82);
  * S, T: oracle/ints.py (libint's one-body engines, libint_iface.cpp:136-190);
    V_ne as the grid quadrature of sum_A Z_A / |r - R_A| (nnuclear.py:15-37);
  * rho = diag(phi^T D phi) (psi_hybrid.py:144-150), F = phi diag(w v) phi^T
    (nwavefunction.cpp:77-107, 161-197): oracle.density / oracle.quadrature;
  * Coulomb potentials: the Poisson driver of poisson_solver.py:18-118 with
    solve_ode2 (ode2.py:35-118) and eval_decomposition_grid
    (evaluate.cpp:129-220), here for many densities at once (poisson_many:
    the Hermite-FEM matrix of an (atom, l) does not depend on m or on the
    density, so it is LU-factored once and solved for every column; checked
    against the per-(l, m) spsolve restatement in tests/test_scf_oracle.py);
  * exchange from orbital-pair potentials, K_mu,nu = sum_i sum_p W phi_mu psi_i
    V[psi_i phi_nu] (the occupied-pair Poisson solves of psi_numeric.py:186-215
    in the AO basis);
  * the SCF step of wavefunction.cpp:64-116 (F C = S C e through S^-1/2,
    D = eta C_occ C_occ^T, E), Pulay DIIS on FDS - SDF (libint_iface.cpp:
    1435-1451 names the method; 6 vectors), core-Hamiltonian guess, and the
    multi-species loop of scf.py:146-273 with the coupling of
    psi_hybrid.py:81-110 (one Becke grid for both species).

The sequence of operations is the one napmo_b200/scf.py runs on the device
(GridRHF, GridAPMO), so that converged energies and iteration counts can be
compared: same guess, same DIIS, same stopping rule (|dE| < tol and
max |X^T (FDS - SDF) X| < 1e-4).
"""
import numpy as np
import scipy.linalg
from threadpoolctl import threadpool_limits

import oracle as O
import ints as OI
import xc as OX

PROTON_MASS = 1836.15267247      # electron masses (napmo/data/constants.py)
BOHR = 0.52917724924             # napmo/data/constants.py

# species constants (napmo/data/elementary_particles.json, coupling_constants.json)
ELECTRON = dict(eta=2.0, charge=-1.0)
NUCLEUS = dict(eta=1.0, charge=1.0)

# even-tempered 5s5p nuclear basis, exponents 4..64 bohr^-2 (ratio 2)
NUCLEAR_5S5P = [(0, [z], [1.0]) for z in (4.0, 8.0, 16.0, 32.0, 64.0)] + \
               [(1, [z], [1.0]) for z in (4.0, 8.0, 16.0, 32.0, 64.0)]


def lebedev_lmax(nang):
    """lebedev_get_order(nang) // 2 (psi_numeric.py:66, lebedev.py:25-31)."""
    orders = {6: 3, 14: 5, 26: 7, 38: 9, 50: 11, 74: 13, 86: 15, 110: 17, 146: 19, 170: 21,
              194: 23, 230: 25, 266: 27, 302: 29, 350: 31, 434: 35, 590: 41, 770: 47,
              974: 53, 1202: 59}
    return orders[nang] // 2


# ------------------------------------------------------------------ Poisson
class PoissonPlan(object):
    """Per-atom tables of poisson_solver.py for one grid and lmax: the radial
    Jacobians, the source matrix of the Hermite FEM right-hand side and the LU
    factors of every (atom, l) system (build_ode2 with the boundary rows of
    V(r_min) and V(r_max))."""

    def __init__(self, grid, lmax):
        self.grid, self.lmax = grid, lmax
        self.atoms = []
        done = {}   # atoms of one element share their radial tables
        for atom in grid.atoms:
            key = (atom.radii, atom.nrad)
            if key in done:
                self.atoms.append(done[key])
                continue
            n = atom.nrad
            r = atom.r
            j1, j2, j3 = O.radial_derivs(n, atom.radii)
            r2, r3 = r * r, r * r * r
            b_y, b_dx = 2 / r, -2 / r2
            j1sq = j1 * j1
            by_new = j1 * b_y - j2 / j1
            bd_new = j2 * b_y + j1sq * b_dx + (j2 * j2 - j1 * j3) / j1sq
            merge = lambda u, v: np.ascontiguousarray(np.array([u, v]).T.ravel())
            bcs = np.array([0.0, np.nan, 0.0, np.nan])
            # right-hand side = Ov2 @ f (rows of the boundary conditions
            # replaced), read off build_ode2 column by column
            ov2 = np.zeros((2 * n, 2 * n))
            zero = np.zeros(2 * n)
            for c in range(2 * n):
                e = np.zeros(2 * n)
                e[c] = 1.0
                coeffs = np.zeros((2 * n, 2 * n))
                rhs = np.zeros(2 * n)
                O.lib.orc_build_ode2(zero, zero, e, bcs, coeffs, rhs, n)
                ov2[:, c] = rhs
            lu = []
            for l in range(lmax + 1):
                l2l = l * (l + 1)
                a_y, a_dx = -l2l / r2, 2 * l2l / r3
                ay_new = a_y * j1sq
                ad_new = (a_dx * j1sq + 2 * a_y * j2) * j1
                coeffs = np.zeros((2 * n, 2 * n))
                rhs = np.zeros(2 * n)
                O.lib.orc_build_ode2(merge(by_new, bd_new), merge(ay_new, ad_new), zero, bcs,
                                     coeffs, rhs, n)
                lu.append(scipy.linalg.lu_factor(coeffs))
            done[key] = dict(n=n, j1=j1, j2=j2, j1sq=j1sq, ov2=ov2, lu=lu)
            self.atoms.append(done[key])


def poisson_many(plan, dens, points=None):
    """V_H of k densities on the grid: dens [k][N] -> V [k][N]
    (poisson_solver.py:18-118 + eval_decomposition_grid for each), or at
    `points` [P][3] only -> V [k][P].  The small LAPACK/BLAS calls run on one
    thread: the OpenMP loops of the C parts use the cores, and BLAS threads
    competing with them cost 4x here."""
    with threadpool_limits(limits=1, user_api='blas'):
        return _poisson_many(plan, dens, points)


def _poisson_many(plan, dens, points):
    grid, lmax = plan.grid, plan.lmax
    dens = np.atleast_2d(np.asarray(dens, dtype=np.float64))
    k, N = dens.shape
    lsize = (lmax + 1) ** 2
    src = np.ascontiguousarray(dens * grid.becke)
    pts = grid.points if points is None else np.ascontiguousarray(points, dtype=np.float64)
    P = pts.shape[0]
    V = np.zeros((k, P))
    PI_4 = 4.0 * np.pi
    off = 0
    for ia, atom in enumerate(grid.atoms):
        A = plan.atoms[ia]
        n = A['n']
        f = np.ascontiguousarray(src[:, off:off + atom.size])
        sph = np.zeros((k * n, lsize))
        O.lib.orc_spherical_expansion_many(atom.nrad, atom.nang, atom.points, atom.weights,
                                           atom.center, k, f, atom.size, lmax, sph)
        sph = sph.reshape(k, n, lsize)
        y = np.zeros((k, lsize, n))
        dt = np.zeros((k, lsize, n))
        r, wr = atom.r, atom.wr
        for l in range(lmax + 1):
            c0, c1 = l * l, (l + 1) * (l + 1)
            aux = np.ascontiguousarray(sph[:, :, c0:c1].transpose(0, 2, 1).reshape(-1, n))
            ncol = aux.shape[0]
            rho_dt = np.zeros_like(aux)
            O.lib.orc_spline_dt_many(aux, rho_dt, n, ncol)
            rho_dx = rho_dt / A['j1']
            fy = -PI_4 * aux
            fd = -PI_4 * rho_dx
            V_rmax = (aux * r ** l * wr).sum(axis=1) * (1.0 / r[-1] ** (l + 1) / (2 * l + 1))
            V_rmin = (aux * r ** (-l - 1) * wr).sum(axis=1) * (r[0] ** l / (2 * l + 1))
            fy_new = fy * A['j1sq']
            fd_new = (fd * A['j1sq'] + 2 * fy * A['j2']) * A['j1']
            fm = np.empty((2 * n, ncol))
            fm[0::2] = fy_new.T
            fm[1::2] = fd_new.T
            rhs = A['ov2'] @ fm
            rhs[0] = V_rmin
            rhs[2 * n - 2] = V_rmax
            sol = scipy.linalg.lu_solve(A['lu'][l], rhs)
            y[:, c0:c1, :] = sol[0::2].T.reshape(k, c1 - c0, n)
            dt[:, c0:c1, :] = ((sol[1::2] / A['j1'][:, None]) * A['j1'][:, None]).T.reshape(
                k, c1 - c0, n)
        O.lib.orc_eval_decomposition_many(0, atom.radii, 0.0, n, lsize, k,
                                          y.reshape(k * lsize, n), dt.reshape(k * lsize, n),
                                          atom.center, P, pts, V, P)
        off += atom.size
    return V


# ------------------------------------------------------------------ systems
def _diis(Fs, errs):
    m = len(Fs)
    B = np.empty((m + 1, m + 1))
    for a in range(m):
        for b in range(a + 1):
            B[a, b] = B[b, a] = sum(float((ea * eb).sum()) for ea, eb in zip(errs[a], errs[b]))
    B[m, :m] = -1.0
    B[:m, m] = -1.0
    B[m, m] = 0.0
    rhs = np.zeros(m + 1)
    rhs[m] = -1.0
    c = np.linalg.solve(B, rhs)
    return [sum(c[a] * Fs[a][s] for a in range(m)) for s in range(len(Fs[0]))]


def nuclear_repulsion(charges):
    E = 0.0
    for i, (Za, Ra) in enumerate(charges):
        for Zb, Rb in charges[:i]:
            E += Za * Zb / np.linalg.norm(np.asarray(Ra) - np.asarray(Rb))
    return E


class Species(object):
    """One species on the grid: phi [n][N], S, H = T / mass + q V[classical
    charges] (grid quadrature), S^-1/2, occupation, eta, charge."""

    def __init__(self, grid, fb, consts, nocc, charges, mass=1.0):
        self.fb = fb
        self.phi = np.ascontiguousarray(O.basis_compute(fb, grid.points).T)
        self.n = self.phi.shape[0]
        self.q, self.eta, self.nocc = consts['charge'], consts['eta'], nocc
        S, T, _ = OI.one_body(fb, [])
        self.S = S
        H = T / mass
        if charges:
            vn = O.nuclear_potential(grid.points, charges)
            H = H + O.quadrature(self.phi, self.q * vn, grid.becke, grid.weights)
        self.H = H
        s, U = np.linalg.eigh(S)
        self.X = U @ np.diag(1.0 / np.sqrt(s)) @ U.T

    def diag(self, F):
        e, Cp = np.linalg.eigh(self.X.T @ F @ self.X)
        C = self.X @ Cp
        Cocc = C[:, :self.nocc]
        return e, C, self.eta * Cocc @ Cocc.T

    def error(self, F, D):
        return self.X.T @ (F @ D @ self.S - self.S @ D @ F) @ self.X


def _centers(atoms):
    return [np.array(xyz, dtype=np.float64) / BOHR for _, xyz in atoms]


class GridRHF(object):
    """Closed-shell SCF of the electrons on the Becke grid (restates
    napmo_b200.scf.GridRHF with exchange 'hf' or 'none')."""

    def __init__(self, atoms, library, elements, nrad=50, nang=110, lmax=None, basis='CC-PVDZ',
                 exchange='hf', diis=6):
        centers = _centers(atoms)
        syms = [s for s, _ in atoms]
        self.grid = O.Grid(centers, [elements[s]['atomic_radii'] for s in syms], nrad, nang)
        self.lmax = lebedev_lmax(nang) if lmax is None else lmax
        self.plan = PoissonPlan(self.grid, self.lmax)
        charges = [(elements[s]['atomic_number'], c) for s, c in zip(syms, centers)]
        nel = sum(z for z, _ in charges)
        fb = O.flat_basis(centers, syms, library, basis)
        self.e = Species(self.grid, fb, ELECTRON, nel // 2, charges)
        self.Enn = nuclear_repulsion(charges)
        self.W = self.grid.becke * self.grid.weights
        self.exchange = exchange
        self.ndiis = diis

    def coulomb(self, rho):
        return poisson_many(self.plan, rho[None, :])[0]

    def exchange_matrix(self, Cocc):
        phi = self.e.phi
        psi = Cocc.T @ phi
        K = np.zeros((self.e.n, self.e.n))
        for i in range(psi.shape[0]):
            V = poisson_many(self.plan, psi[i] * phi)
            K += (phi * (self.W * psi[i])) @ V.T
        return 0.5 * (K + K.T)

    def fock(self, D, Cocc):
        sp, g = self.e, self.grid
        rho = O.density(sp.phi, D)
        vH = self.coulomb(rho)
        F = sp.H + O.quadrature(sp.phi, vH, g.becke, g.weights)
        if self.exchange == 'hf':
            F = F - self.exchange_matrix(Cocc)
        return F, 0.5 * float((D * (sp.H + F)).sum()), rho, vH

    def iterations(self, maxiter=100, tol=1e-8):
        """The SCF one iteration at a time: yields (iteration, E, max error,
        converged, D) after each Fock build; stops after convergence."""
        sp = self.e
        _, C, D = sp.diag(sp.H)
        Cocc = C[:, :sp.nocc]
        Fs, errs = [], []
        E_prev = None
        for it in range(1, maxiter + 1):
            F, Eel, rho, vH = self.fock(D, Cocc)
            E = Eel + self.Enn
            err = sp.error(F, D)
            Fs.append((F,))
            errs.append((err,))
            if len(Fs) > self.ndiis:
                Fs.pop(0)
                errs.pop(0)
            emax = float(np.abs(err).max())
            if E_prev is not None and abs(E - E_prev) < tol and emax < 1e-4:
                yield it, E, emax, True, D
                return
            yield it, E, emax, False, D
            E_prev = E
            if len(Fs) > 1:
                F = _diis(Fs, errs)[0]
            _, C, D = sp.diag(F)
            Cocc = C[:, :sp.nocc]

    def run(self, maxiter=100, tol=1e-8):
        history = []
        for it, E, emax, converged, D in self.iterations(maxiter, tol):
            history.append((E, emax))
        return dict(energy=E, iterations=it, converged=converged, history=history, D=D,
                    electrons=float((D * self.e.S).sum()))


class GridAPMO(object):
    """Electrons and one quantum nucleus on one Becke grid (restates
    napmo_b200.scf.GridAPMO with HF exchange):

    E = sum_s tr(D_s H_s) + 1/2 q_e^2 <rho_e|V[rho_e]> - 1/2 tr(D_e K_e)
        + 1/2 q_e q_n (<rho_e|V[rho_n]> + <rho_n|V[rho_e]>) + E_nn(classical)
    (the coupling as nAPMO's 1/2 sum_s tr(D_s J_s), scf.py:494-520)."""

    def __init__(self, atoms, library, elements, quantum=(0,), nrad=100, nang=302, lmax=None,
                 basis='CC-PVDZ', diis=6, mass=PROTON_MASS):
        centers = _centers(atoms)
        syms = [s for s, _ in atoms]
        self.grid = O.Grid(centers, [elements[s]['atomic_radii'] for s in syms], nrad, nang)
        self.lmax = lebedev_lmax(nang) if lmax is None else lmax
        self.plan = PoissonPlan(self.grid, self.lmax)
        classical = [(elements[s]['atomic_number'], c) for i, (s, c) in
                     enumerate(zip(syms, centers)) if i not in quantum]
        nel = sum(elements[s]['atomic_number'] for s in syms)
        fb_e = O.flat_basis(centers, syms, library, basis)
        self.e = Species(self.grid, fb_e, ELECTRON, nel // 2, classical)
        qc = [centers[i] for i in quantum]
        nsym = [syms[i] + '_1' for i in quantum]
        lib_n = {'NUCLEAR-5S5P': {s: NUCLEAR_5S5P for s in nsym}}
        fb_n = O.flat_basis(qc, nsym, lib_n, 'NUCLEAR-5S5P')
        self.nuc = Species(self.grid, fb_n, NUCLEUS, len(quantum), classical, mass=mass)
        self.quantum_centers = qc
        self.Enn = nuclear_repulsion(classical)
        self.W = self.grid.becke * self.grid.weights
        self.ndiis = diis

    def exchange_matrix(self, Cocc):
        sp = self.e
        psi = Cocc.T @ sp.phi
        K = np.zeros((sp.n, sp.n))
        for i in range(psi.shape[0]):
            V = poisson_many(self.plan, psi[i] * sp.phi)
            K += (sp.phi * (self.W * psi[i])) @ V.T
        return 0.5 * (K + K.T)

    def fock(self, De, Dn, Ce):
        e, n, g = self.e, self.nuc, self.grid
        qq = e.q * n.q
        rho_e = O.density(e.phi, De)
        rho_n = O.density(n.phi, Dn)
        V = poisson_many(self.plan, np.stack([rho_e, rho_n]))
        v_e, v_n = V[0], V[1]
        Fe = e.H + O.quadrature(e.phi, e.q * e.q * v_e + qq * v_n, g.becke, g.weights)
        K = self.exchange_matrix(Ce[:, :e.nocc])
        Fe = Fe - K
        Fn = n.H + O.quadrature(n.phi, qq * v_e, g.becke, g.weights)
        E_J = 0.5 * e.q * e.q * float((self.W * rho_e * v_e).sum())
        E_K = -0.5 * float((De * K).sum())
        coup = 0.5 * qq * (float((self.W * rho_e * v_n).sum()) +
                           float((self.W * rho_n * v_e).sum()))
        E = (float((De * e.H).sum()) + E_J + E_K + float((Dn * n.H).sum()) + coup + self.Enn)
        return Fe, Fn, E, (rho_e, rho_n, v_e, v_n)

    def guess(self):
        """Electrons with the quantum nuclei as unit point charges, then the
        nucleus in that electron density's field."""
        e, n, g = self.e, self.nuc, self.grid
        qq = e.q * n.q
        vq = O.nuclear_potential(g.points, [(1.0, c) for c in self.quantum_centers])
        _, Ce, De = e.diag(e.H + O.quadrature(e.phi, qq * vq, g.becke, g.weights))
        v_e = poisson_many(self.plan, O.density(e.phi, De)[None, :])[0]
        _, Cn, Dn = n.diag(n.H + O.quadrature(n.phi, qq * v_e, g.becke, g.weights))
        return Ce, De, Cn, Dn

    def run(self, maxiter=100, tol=1e-8):
        e, n = self.e, self.nuc
        Ce, De, Cn, Dn = self.guess()
        Fs, errs, history = [], [], []
        E_prev, converged = None, False
        for it in range(1, maxiter + 1):
            Fe, Fn, E, _ = self.fock(De, Dn, Ce)
            err_e, err_n = e.error(Fe, De), n.error(Fn, Dn)
            Fs.append((Fe, Fn))
            errs.append((err_e, err_n))
            if len(Fs) > self.ndiis:
                Fs.pop(0)
                errs.pop(0)
            emax = (float(np.abs(err_e).max()), float(np.abs(err_n).max()))
            history.append((E,) + emax)
            if E_prev is not None and abs(E - E_prev) < tol and max(emax) < 1e-4:
                converged = True
                break
            E_prev = E
            if len(Fs) > 1:
                Fe, Fn = _diis(Fs, errs)
            _, Ce, De = e.diag(Fe)
            _, Cn, Dn = n.diag(Fn)
        return dict(energy=E, iterations=it, converged=converged, history=history, De=De, Dn=Dn,
                    electrons=float((De * e.S).sum()), nuclei=float((Dn * n.S).sum()))


def spin_occupations(nelectron, multiplicity=None):
    """(n_alpha, n_beta) as nAPMO splits e- (molecular_system.py:214-290)."""
    if not multiplicity:
        multiplicity = (nelectron % 2) + 1
    unpaired = multiplicity - 1
    left = nelectron - unpaired
    if left < 0 or left % 2 != 0:
        raise ValueError('Bad charge / multiplicity')
    return left // 2 + unpaired, left // 2


class GridMultiSCF(object):
    """Unrestricted grid SCF (restates napmo_b200.scf.GridMultiSCF): e-alpha
    and e-beta species (eta = 1, nAPMO's 'uhf' split) and optionally one
    quantum nucleus on one Becke grid; Coulomb between all species, HF
    exchange within each spin species, no self-interaction of the nucleus."""

    def __init__(self, atoms, library, elements, quantum=(), nrad=50, nang=110, lmax=None,
                 basis='CC-PVDZ', charge=0, multiplicity=None, diis=6, mass=PROTON_MASS,
                 exchange='hf'):
        centers = _centers(atoms)
        syms = [s for s, _ in atoms]
        self.grid = O.Grid(centers, [elements[s]['atomic_radii'] for s in syms], nrad, nang)
        self.lmax = lebedev_lmax(nang) if lmax is None else lmax
        self.plan = PoissonPlan(self.grid, self.lmax)
        classical = [(elements[s]['atomic_number'], c) for i, (s, c) in
                     enumerate(zip(syms, centers)) if i not in quantum]
        nel = sum(elements[s]['atomic_number'] for s in syms) - int(charge)
        na, nb = spin_occupations(nel, multiplicity)
        fb_e = O.flat_basis(centers, syms, library, basis)
        spin = dict(eta=1.0, charge=-1.0)
        self.species = [Species(self.grid, fb_e, spin, na, classical),
                        Species(self.grid, fb_e, spin, nb, classical)]
        self.is_electron = [True, True]
        self.quantum_centers = [centers[i] for i in quantum]
        if quantum:
            nsym = [syms[i] + '_1' for i in quantum]
            lib_n = {'NUCLEAR-5S5P': {s: NUCLEAR_5S5P for s in nsym}}
            fb_n = O.flat_basis(self.quantum_centers, nsym, lib_n, 'NUCLEAR-5S5P')
            self.species.append(Species(self.grid, fb_n, NUCLEUS, len(quantum), classical,
                                        mass=mass))
            self.is_electron.append(False)
        self.Enn = nuclear_repulsion(classical)
        self.W = self.grid.becke * self.grid.weights
        self.exchange = exchange
        self.ndiis = diis

    def _exchange(self, sp, Cocc):
        psi = Cocc.T @ sp.phi
        K = np.zeros((sp.n, sp.n))
        for i in range(psi.shape[0]):
            V = poisson_many(self.plan, psi[i] * sp.phi)
            K += (sp.phi * (self.W * psi[i])) @ V.T
        return 0.5 * (K + K.T)

    def fock(self, Ds, Cs):
        sps, g = self.species, self.grid
        rhos = [O.density(sp.phi, D) for sp, D in zip(sps, Ds)]
        vs = poisson_many(self.plan, np.stack(rhos))
        Fs, E = [], self.Enn
        vxc = [None] * len(sps)
        if self.exchange == 'lda':   # spin-polarised LDA of the two spin densities
            zx, xa, xb = OX.lda_x_polarized(rhos[0], rhos[1])
            zc, ca, cb = OX.lda_c_vwn_polarized(rhos[0], rhos[1])
            vxc[0], vxc[1] = xa + ca, xb + cb
            E += float((self.W * (rhos[0] + rhos[1]) * (zx + zc)).sum())
        for s, sp in enumerate(sps):
            pot = np.zeros(g.size)
            for u, (tp, v) in enumerate(zip(sps, vs)):
                if u == s and not self.is_electron[s]:
                    continue
                pot = pot + (sp.q * tp.q) * v
            F = sp.H + O.quadrature(sp.phi, pot if vxc[s] is None else pot + vxc[s], g.becke,
                                    g.weights)
            E += float((Ds[s] * sp.H).sum()) + 0.5 * float((self.W * rhos[s] * pot).sum())
            if self.exchange == 'hf' and self.is_electron[s] and sp.nocc > 0:
                K = self._exchange(sp, Cs[s][:, :sp.nocc])
                F = F - K
                E -= 0.5 * float((Ds[s] * K).sum())
            Fs.append(F)
        return Fs, E

    def guess(self):
        sps, g = self.species, self.grid
        H = sps[0].H
        if len(sps) > 2:
            vq = O.nuclear_potential(g.points, [(1.0, c) for c in self.quantum_centers])
            H = H + O.quadrature(sps[0].phi, sps[0].q * sps[2].q * vq, g.becke, g.weights)
        Cs, Ds = [], []
        for sp in sps[:2]:
            _, C, D = sp.diag(H)
            Cs.append(C)
            Ds.append(D)
        if len(sps) > 2:
            nuc = sps[2]
            v_e = poisson_many(self.plan, O.density(sps[0].phi, Ds[0] + Ds[1])[None, :])[0]
            _, C, D = nuc.diag(nuc.H + O.quadrature(nuc.phi, sps[0].q * nuc.q * v_e, g.becke,
                                                    g.weights))
            Cs.append(C)
            Ds.append(D)
        return Cs, Ds

    def run(self, maxiter=100, tol=1e-8):
        sps = self.species
        Cs, Ds = self.guess()
        Fh, errs, history = [], [], []
        E_prev, converged = None, False
        for it in range(1, maxiter + 1):
            Fs, E = self.fock(Ds, Cs)
            err = [sp.error(F, D) for sp, F, D in zip(sps, Fs, Ds)]
            Fh.append(tuple(Fs))
            errs.append(tuple(err))
            if len(Fh) > self.ndiis:
                Fh.pop(0)
                errs.pop(0)
            emax = tuple(float(np.abs(x).max()) for x in err)
            history.append((E,) + emax)
            if E_prev is not None and abs(E - E_prev) < tol and max(emax) < 1e-4:
                converged = True
                break
            E_prev = E
            if len(Fh) > 1:
                Fs = _diis(Fh, errs)
            Cs, Ds = [], []
            for sp, F in zip(sps, Fs):
                _, C, D = sp.diag(F)
                Cs.append(C)
                Ds.append(D)
        return dict(energy=E, iterations=it, converged=converged, history=history, D=Ds,
                    alpha=float((Ds[0] * sps[0].S).sum()), beta=float((Ds[1] * sps[1].S).sum()))
