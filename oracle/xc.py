"""CPU restatement of the local functionals of nAPMO's grid path (test
infrastructure only).

nAPMO takes its electronic functionals from LibXC through pylibxc
(napmo/functional/xc_interface.py:29-90: 'lda' = lda_x + lda_c_vwn,
unpolarised), a third-party library absent here; its published forms are
restated: Dirac-Slater exchange and the Vosko-Wilk-Nusair paramagnetic
correlation fit (VWN5, Can. J. Phys. 58, 1200 (1980)), which is what LibXC's
lda_c_vwn evaluates.  Pinned against nAPMO's own fixtures
(napmo/functional/test/*.txt, subsampled into tests/golden/xc_lda.npz).
The electron-proton correlation epc17-2 restates
napmo/functional/interspecies_correlation.py:36-68.
"""
import numpy as np

# densities below this give zk = vrho = 0 (nAPMO's fixtures, produced through
# LibXC, place the cut between 3.1e-25 and 1.2e-22)
DENS_CUT = 1e-24

CX = -(3.0 / np.pi) ** (1.0 / 3.0)       # v_x = CX rho^(1/3)
VWN_A, VWN_B, VWN_C, VWN_X0 = 0.0310907, 3.72744, 12.9352, -0.10498


def lda_x(rho):
    """(zk, vrho) of Dirac-Slater exchange, per particle and its derivative."""
    rho = np.asarray(rho, np.float64)
    m = rho >= DENS_CUT
    r13 = np.cbrt(np.where(m, rho, 0.0))
    return np.where(m, 0.75 * CX * r13, 0.0), np.where(m, CX * r13, 0.0)


# spin-polarised VWN5: the ferromagnetic fit and the spin stiffness
# (Vosko, Wilk, Nusair 1980, the parameters LibXC's lda_c_vwn uses)
VWN_F = (0.01554535, 7.06042, 18.0578, -0.32500)
VWN_ALPHA = (-1.0 / (6.0 * np.pi ** 2), 1.13107, 13.0045, -0.0047584)
FZ_DEN = 2.0 ** (4.0 / 3.0) - 2.0           # f(z) = ((1+z)^4/3 + (1-z)^4/3 - 2) / FZ_DEN
FPP0 = 4.0 / (9.0 * (2.0 ** (1.0 / 3.0) - 1.0))  # f''(0)


def _vwn_fit(x, A, b, c, x0):
    """(G, dG/dx) of the VWN interpolation at x = sqrt(r_s)."""
    X = x * x + b * x + c
    X0 = x0 * x0 + b * x0 + c
    Q = np.sqrt(4.0 * c - b * b)
    at = np.arctan(Q / (2.0 * x + b))
    g = A * (np.log(x * x / X) + 2.0 * b / Q * at
             - b * x0 / X0 * (np.log((x - x0) ** 2 / X) + 2.0 * (b + 2.0 * x0) / Q * at))
    dX = 2.0 * x + b
    den = dX * dX + Q * Q
    dg = A * (2.0 / x - dX / X - 4.0 * b / den
              - b * x0 / X0 * (2.0 / (x - x0) - dX / X - 4.0 * (b + 2.0 * x0) / den))
    return g, dg


def lda_x_polarized(rho_a, rho_b):
    """(zk, v_a, v_b) of spin-polarised Dirac-Slater exchange:
    e_x = -3/4 (6/pi)^(1/3) (rho_a^(4/3) + rho_b^(4/3)), zk = e_x / rho,
    v_s = -(6 rho_s / pi)^(1/3); zero where rho_a + rho_b < DENS_CUT
    (negative spin densities count as zero)."""
    ra = np.maximum(np.asarray(rho_a, np.float64), 0.0)
    rb = np.maximum(np.asarray(rho_b, np.float64), 0.0)
    rho = ra + rb
    m = rho >= DENS_CUT
    c = -np.cbrt(6.0 / np.pi)
    a13, b13 = np.cbrt(ra), np.cbrt(rb)
    e = 0.75 * c * (ra * a13 + rb * b13)
    zk = np.where(m, e / np.where(m, rho, 1.0), 0.0)
    return zk, np.where(m, c * a13, 0.0), np.where(m, c * b13, 0.0)


def lda_c_vwn_polarized(rho_a, rho_b):
    """(zk, v_a, v_b) of spin-polarised VWN5 correlation:
    e_c(r_s, z) = e_P + a_c f(z) / f''(0) (1 - z^4) + (e_F - e_P) f(z) z^4,
    v_s = e_c - (r_s / 3) de_c/dr_s + (s - z) de_c/dz (s = +1 for alpha,
    -1 for beta); zero where rho_a + rho_b < DENS_CUT."""
    ra = np.maximum(np.asarray(rho_a, np.float64), 0.0)
    rb = np.maximum(np.asarray(rho_b, np.float64), 0.0)
    rho = ra + rb
    m = rho >= DENS_CUT
    r = np.where(m, rho, 1.0)
    z = np.clip(np.where(m, (ra - rb) / r, 0.0), -1.0, 1.0)
    x = np.sqrt(np.cbrt(3.0 / (4.0 * np.pi * r)))
    eP, dP = _vwn_fit(x, VWN_A, VWN_B, VWN_C, VWN_X0)
    eF, dF = _vwn_fit(x, *VWN_F)
    ac, dac = _vwn_fit(x, *VWN_ALPHA)
    zp, zm = np.cbrt(1.0 + z), np.cbrt(1.0 - z)
    f = ((1.0 + z) * zp + (1.0 - z) * zm - 2.0) / FZ_DEN
    df = (4.0 / 3.0) * (zp - zm) / FZ_DEN
    z3 = z * z * z
    z4 = z3 * z
    ec = eP + ac * f / FPP0 * (1.0 - z4) + (eF - eP) * f * z4
    dx = dP + dac * f / FPP0 * (1.0 - z4) + (dF - dP) * f * z4
    dz = ac / FPP0 * (df * (1.0 - z4) - 4.0 * z3 * f) + (eF - eP) * (df * z4 + 4.0 * z3 * f)
    base = ec - x / 6.0 * dx
    return (np.where(m, ec, 0.0), np.where(m, base + (1.0 - z) * dz, 0.0),
            np.where(m, base - (1.0 + z) * dz, 0.0))


def lda_c_vwn(rho):
    """(zk, vrho) of VWN5 correlation (paramagnetic)."""
    rho = np.asarray(rho, np.float64)
    m = rho >= DENS_CUT
    r = np.where(m, rho, 1.0)
    A, b, c, x0 = VWN_A, VWN_B, VWN_C, VWN_X0
    x = np.sqrt(np.cbrt(3.0 / (4.0 * np.pi * r)))      # sqrt(r_s)
    X = x * x + b * x + c
    X0 = x0 * x0 + b * x0 + c
    Q = np.sqrt(4.0 * c - b * b)
    at = np.arctan(Q / (2.0 * x + b))
    ec = A * (np.log(x * x / X) + 2.0 * b / Q * at
              - b * x0 / X0 * (np.log((x - x0) ** 2 / X) + 2.0 * (b + 2.0 * x0) / Q * at))
    dX = 2.0 * x + b
    den = dX * dX + Q * Q
    dec = A * (2.0 / x - dX / X - 4.0 * b / den
               - b * x0 / X0 * (2.0 / (x - x0) - dX / X - 4.0 * (b + 2.0 * x0) / den))
    vc = ec - x / 6.0 * dec                              # v = e - (r_s / 3) de/dr_s
    return np.where(m, ec, 0.0), np.where(m, vc, 0.0)


def epc17_2(rhoE, rhoN):
    """(energy per electron, potential of the electrons, of the nuclei) of
    epc17-2 at common points; if any density is below 1e-200 every point
    uses the alternative potentials, as nAPMO does."""
    # negative densities (rounding) count as zero, as in the library's kernel
    # (nAPMO's own numpy code returns NaN there)
    rhoE = np.maximum(np.asarray(rhoE, np.float64), 0.0)
    rhoN = np.maximum(np.asarray(rhoN, np.float64), 0.0)
    a, b, c = 2.35, 2.4, 6.6
    den = a - b * np.sqrt(rhoE * rhoN) + c * rhoE * rhoN
    ene = -rhoN / den
    if np.any(np.abs(rhoE) < 1.0e-200) or np.any(np.abs(rhoN) < 1.0e-200):
        pa = (b * np.sqrt(rhoE) * rhoN ** 1.5 - 2.0 * a * rhoN) / den ** 2 / 2.0
        pb = (b * np.sqrt(rhoN) * rhoE ** 1.5 - 2.0 * a * rhoE) / den ** 2 / 2.0
    else:
        s = np.sqrt(rhoE * rhoN)
        pa = (rhoE * rhoN * (c * rhoN - b * rhoN / (2.0 * s)) - rhoN * den) / den ** 2
        pb = (rhoN * rhoE * (c * rhoE - b * rhoE / (2.0 * s)) - rhoE * den) / den ** 2
    return ene, pa, pb
