"""CPU restatement of nAPMO's numerical-orbital operators (test
infrastructure only): the radial second derivative, the kinetic operator on
the grid and the Becke-Dickson orbital correction.

* ``deriv2``          napmo/grids/radial.py, src/grid/radial.cpp:51-192
* ``compute_kinetic`` napmo/wavefunction/nkinetic.py:15-73
* ``compute_dpsi``    napmo/wavefunction/ndpsi.py:15-89 (A. D. Becke and
                      R. M. Dickson, J. Chem. Phys. 92, 3610 (1990))

``deriv2`` is pinned by the vectors of napmo/wavefunction/test/test_kinetic.py
(tests/golden/known_answers.json); the other two are built from the oracle's
projection, spline, FEM and multipole-evaluation restatements (oracle.py),
which are pinned against nAPMO's compiled sources.
"""
import numpy as np

import oracle as O

# Standard finite-difference weights on a unit-spaced axis (the tables of
# B. Fornberg, Math. Comp. 51, 699 (1988)), as exact fractions over a common
# denominator.  One-sided 7-point stencils at nodes 0..3 of nodes 0..6:
_D1_EDGE = np.array([[-1764, 4320, -5400, 4800, -2700, 864, -120],
                     [-120, -924, 1800, -1200, 600, -180, 24],
                     [24, -288, -420, 960, -360, 96, -12],
                     [-12, 108, -540, 0, 540, -108, 12]], np.float64)   # / 720
_D2_EDGE = np.array([[1624, -6264, 10530, -10160, 5940, -1944, 274],
                     [274, -294, -510, 940, -570, 186, -26],
                     [-26, 456, -840, 400, 30, -24, 4],
                     [4, -54, 540, -980, 540, -54, 4]], np.float64)   # / 360
# centred 9-point stencils (nodes -4..4)
_D1_MID = np.array([144, -1536, 8064, -32256, 0, 32256, -8064, 1536, -144],
                   np.float64)   # / 40320
_D2_MID = np.array([-36, 512, -4032, 32256, -57400, 32256, -4032, 512, -36],
                   np.float64)   # / 20160


def deriv2(r, radii, f):
    """(1/r) d2/dr2 (r f) on the Chebyshev grid r = radii (1+cos w)/(1-cos w),
    w_k = (k+1) pi/(n+1), r ascending (r[n-1-k] <-> w_k)."""
    f = np.asarray(f, np.float64)
    n = f.shape[0]
    assert n >= 8
    H = np.pi / (n + 1.0)
    g = f[::-1]                       # g[k] = f(w_k)
    d1, d2 = np.zeros(n), np.zeros(n)
    for i in range(4):
        d1[i] = (_D1_EDGE[i] @ g[:7]) / (720.0 * H)
        d2[i] = (_D2_EDGE[i] @ g[:7]) / (360.0 * H * H)
        j = n - 1 - i                  # mirror image at the far end
        d1[j] = -(_D1_EDGE[i] @ g[::-1][:7]) / (720.0 * H)
        d2[j] = (_D2_EDGE[i] @ g[::-1][:7]) / (360.0 * H * H)
    for i in range(4, n - 4):
        d1[i] = (_D1_MID @ g[i - 4:i + 5]) / (40320.0 * H)
        d2[i] = (_D2_MID @ g[i - 4:i + 5]) / (20160.0 * H * H)
    w = (np.arange(n) + 1) * H
    X, Y = np.cos(w), np.sin(w)
    q = 1.0 - X
    wr = -q * q / (2.0 * radii * Y)                                   # dw/dr
    wrr = q ** 3 * (2.0 * Y * Y - q * X) / (4.0 * radii ** 2 * Y ** 3)  # d2w/dr2
    rr = np.asarray(r, np.float64)[::-1]
    out = wr * wr * d2 + (wrr + 2.0 * wr / rr) * d1
    return out[::-1].copy()


def _tail_splines(atom, vals):
    """(y [lsize][n], dt [lsize][n]) splines of radial columns vals [n][lsize]."""
    ys = np.ascontiguousarray(vals.T)
    dts = np.array([O._spline_dt(np.ascontiguousarray(y)) for y in ys])
    return ys, dts


def compute_kinetic(grid, psi, lmax):
    """-1/2 laplacian of psi at every grid point (nkinetic.py:15-73)."""
    out = np.zeros(grid.size)
    off = 0
    for a, atom in enumerate(grid.atoms):
        p = psi[off:off + atom.size] * grid.becke[off:off + atom.size]
        sph = O.spherical_expansion(atom, p, lmax)
        r = atom.r
        vals = np.zeros_like(sph)
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                idx = l * l + m + l
                aux = sph[:, idx].copy()
                vals[:, idx] = deriv2(r, atom.radii, aux) - l * (l + 1) / (r * r) * aux
        O.evaluate_decomposition(grid, a, _tail_splines(atom, vals), out)
        off += atom.size
    return -0.5 * out


def spherical_average(atom, f):
    """Per radial shell: sum_j f_j w_j / sum_j w_j (AtomicGrid.spherical_average)."""
    nang = atom.nang
    fw = (f * atom.weights).reshape(atom.nrad, nang).sum(axis=1)
    return fw / atom.weights.reshape(atom.nrad, nang).sum(axis=1)


def compute_dpsi(grid, lmax, phi, doi, oi, ri, V_tot, mass_inv):
    """Becke-Dickson orbital correction (ndpsi.py:15-89): for every atom and
    (l, m) the Hermite-FEM solution of
        u'' + (2/r) u' + a u = f,   a = -2/m_inv (l(l+1)/r^2 + <V>(r) - e - de),
                                     f = -2/m_inv [(phi de - R) wb]_lm,
    u = 0 at both ends, then summed over atoms at every point."""
    from scipy.sparse import csc_matrix
    from scipy.sparse.linalg import spsolve
    src = (phi * doi - ri) * grid.becke
    out = np.zeros(grid.size)
    off = 0
    for a_i, atom in enumerate(grid.atoms):
        sl = slice(off, off + atom.size)
        sph = O.spherical_expansion(atom, src[sl].copy(), lmax)
        vsph = spherical_average(atom, V_tot[sl] * grid.becke[sl])
        r = atom.r
        n = atom.nrad
        j1, j2, j3 = O.radial_derivs(n, atom.radii)
        b_y, b_dx = 2.0 / r, -2.0 / (r * r)
        ys, dts = [], []
        for l in range(lmax + 1):
            a_y = -2.0 / mass_inv * (l * (l + 1.0) / (r * r) + (vsph - oi - doi))
            a_dx = O._spline_dt(np.ascontiguousarray(a_y)) / j1
            for m in range(-l, l + 1):
                aux = np.ascontiguousarray(sph[:, l * l + m + l])
                mu_dx = O._spline_dt(aux) / j1
                fy = -2.0 / mass_inv * aux
                fd = -2.0 / mass_inv * mu_dx
                j1sq = j1 * j1
                by_new = j1 * b_y - j2 / j1
                bd_new = j2 * b_y + j1sq * b_dx + (j2 * j2 - j1 * j3) / j1sq
                ay_new = a_y * j1sq
                ad_new = (a_dx * j1sq + 2 * a_y * j2) * j1
                fy_new = fy * j1sq
                fd_new = (fd * j1sq + 2 * fy * j2) * j1
                merge = lambda u, v: np.ascontiguousarray(np.array([u, v]).T.ravel())
                bcs = np.array([0.0, np.nan, 0.0, np.nan])
                coeffs = np.zeros((2 * n, 2 * n))
                rhs = np.zeros(2 * n)
                O.lib.orc_build_ode2(merge(by_new, bd_new), merge(ay_new, ad_new),
                                     merge(fy_new, fd_new), bcs, coeffs, rhs, n)
                sol = spsolve(csc_matrix(coeffs), rhs)
                ys.append(sol[::2].copy())
                dts.append((sol[1::2] / j1) * j1)
        O.evaluate_decomposition(grid, a_i, (np.array(ys), np.array(dts)), out)
        off += atom.size
    return out


def becke_scf(grid, phi0, e0, vnuc, lmax, nocc=1, eta=2.0, kappa=-1.0, charge=-1.0, mass_inv=1.0,
              maxiter=100, tol=1e-8, pce=0.0, verbose=False, record=None):
    """The Becke-Dickson SCF of nAPMO's numerical solver for a closed-shell
    species whose occupied orbitals start as the rows of phi0 with energies
    e0 (psi_numeric.py:23-424, psi_optimization.py:124-221, the loop of
    test_psi_numeric_becke_He.py:100-130), with the oracle's operators and
    numpy's generalised eigensolver.  Returns the energy history; with
    `record` (a list) each optimiser step appends its (S, F) of the
    orbitals-plus-corrections space."""
    import scipy.linalg
    ndim = nocc
    x_factor = kappa / eta
    W = grid.becke * grid.weights

    def mat(A, B):
        return (A * W) @ B.T

    def normalize(psi):
        S = mat(psi, psi)
        psi = psi / np.sqrt(S.diagonal())[:, None]
        return psi, mat(psi, psi)

    def one_body(psi):
        Tg = np.array([compute_kinetic(grid, p, lmax) for p in psi]) * mass_inv
        Vg = psi * vnuc * charge
        return Tg, Vg, mat(psi, Tg) + mat(psi, Vg)

    def coul(rho):
        return O.compute_coulomb(grid, rho, lmax)

    def two_body(psi, D):
        Jpot = coul((psi * psi * eta).sum(axis=0))
        G = mat(psi, psi * Jpot)
        aux = {}
        for s in range(ndim):
            for v in range(s + 1):
                aux[(s, v)] = coul(psi[s] * psi[v])
        K = np.array([sum(psi[k] * aux[(max(l, j), min(l, j))] * D[k, l]
                          for k in range(ndim) for l in range(ndim)) for j in range(ndim)])
        E = mat(psi, K)
        E = np.triu(E) + np.triu(E, 1).T
        return Jpot, K, (G + x_factor * E) * charge ** 2

    def iterate(S, F, H, G):
        e, C = scipy.linalg.eigh(F, S)
        D = eta * C[:, :nocc] @ C[:, :nocc].T
        return e, C, D, float((D * (H + 0.5 * G)).sum())

    psi, S = normalize(np.asarray(phi0, dtype=np.float64)[:ndim])
    Tg, Vg, H = one_body(psi)
    _, C = scipy.linalg.eigh(H, S)
    D = eta * C[:, :nocc] @ C[:, :nocc].T
    Jpot, K, G = two_body(psi, D)
    O_, C, D, E = iterate(S, H + G, H, G)
    prev_O = np.asarray(e0, dtype=np.float64)
    history = [E + pce]
    E_prev = 0.0
    for it in range(maxiter):
        # PSIO_BECKE.optimize
        V_tot = Vg + psi * Jpot + K * x_factor
        R = Tg + V_tot - prev_O[:ndim, None] * psi
        de = np.array([float((R[i] * psi[i] * W).sum()) for i in range(ndim)])
        dpsi = np.array([compute_dpsi(grid, lmax, psi[i], de[i], prev_O[i], R[i], V_tot[i],
                                      mass_inv) for i in range(ndim)])
        ext = np.vstack([psi, dpsi])
        m = ext.shape[0]
        Sx = mat(ext, ext)
        Hg = np.array([compute_kinetic(grid, p, lmax) for p in ext]) * mass_inv + ext * vnuc * charge
        pot = {}
        for s in range(m):
            for v in range(s + 1):
                pot[(s, v)] = coul(ext[s] * ext[v])
        Kg = np.array([sum(ext[s] * pot[(max(s, v), min(s, v))] for s in range(m))
                       for v in range(m)])
        Fx = mat(ext, Hg + ext * Jpot - Kg)
        Fx = (Fx + Fx.T) / 2.0
        if record is not None:
            record.append((Sx.copy(), Fx.copy()))
        ex, Cx = scipy.linalg.eigh(Fx, Sx)
        prev_O = O_.copy()
        psi = (Cx.T @ ext)[:ndim]
        # PSIN: normalize, one-body, two-body, Fock, iterate
        psi, S = normalize(psi)
        Tg, Vg, H = one_body(psi)
        Jpot, K, G = two_body(psi, D)
        O_, C, D, E = iterate(S, H + G, H, G)
        history.append(E + pce)
        if verbose:
            print(it + 1, E + pce, abs(E + pce - E_prev))
        if abs(E + pce - E_prev) < tol:
            break
        E_prev = E + pce
    return history
