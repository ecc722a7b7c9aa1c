"""Grid SCF of the electrons (napmo_b200.scf.GridRHF): convergence, electron
count, the closed-shell energy of H2O/cc-pVDZ with grid J and exchange, and
the int8 contractions against FP64 at the converged energy."""
import pytest

from conftest import gpu_available
from helpers import H2O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]


@pytest.mark.parametrize('exchange,lo,hi', [('hf', -76.035, -76.020), ('lda-x', -75.30, -75.10),
                                             ('lda', -75.90, -75.80)])
def test_grid_scf_h2o(exchange, lo, hi):
    from napmo_b200.scf import GridRHF
    from napmo_b200.system import build_system
    r64 = GridRHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange=exchange).run(tol=1e-9)
    assert r64['converged'] and r64['iterations'] <= 30
    assert abs(r64['electrons'] - 10.0) < 1e-8
    assert lo < r64['energy'] < hi
    r8 = GridRHF(build_system(H2O, 'CC-PVDZ'), 50, 110, exchange=exchange,
                 precision='int8x4').run(tol=1e-9)
    assert r8['converged']
    assert abs(r8['energy'] - r64['energy']) <= 1e-6


def test_grid_apmo_hcn():
    """Electrons + quantum H nucleus (5s5p), coupled through the grid."""
    from helpers import HCN
    from napmo_b200.scf import GridAPMO
    from napmo_b200.system import build_system
    res = {}
    for prec in ('fp64', 'int8x4'):
        ms = build_system(HCN, 'CC-PVDZ', quantum=(0,))
        res[prec] = GridAPMO(ms, 'H_1', 50, 110, precision=prec).run(tol=1e-9)
        assert res[prec]['converged'] and res[prec]['iterations'] <= 40
        assert abs(res[prec]['electrons'] - 14.0) < 1e-8
        assert abs(res[prec]['nuclei'] - 1.0) < 1e-8
    assert -93.0 < res['fp64']['energy'] < -92.7
    assert abs(res['int8x4']['energy'] - res['fp64']['energy']) <= 1e-6


def test_grid_apmo_hcn_lda_epc():
    """Electrons with LDA (Slater + VWN5) and the epc17-2 electron-proton
    correlation: converges, the correlation lowers the energy, int8 = FP64."""
    from helpers import HCN
    from napmo_b200.scf import GridAPMO
    from napmo_b200.system import build_system
    res = {}
    for corr in (None, 'epc17-2'):
        for prec in ('fp64', 'int8x4'):
            ms = build_system(HCN, 'CC-PVDZ', quantum=(0,))
            r = GridAPMO(ms, 'H_1', 50, 110, precision=prec, exchange='lda',
                         correlation=corr).run(tol=1e-9)
            assert r['converged'] and abs(r['electrons'] - 14.0) < 1e-8
            res[(corr, prec)] = r['energy']
        assert abs(res[(corr, 'int8x4')] - res[(corr, 'fp64')]) <= 1e-6
    assert -92.7 < res[(None, 'fp64')] < -92.5
    assert -0.1 < res[('epc17-2', 'fp64')] - res[(None, 'fp64')] < 0.0


def _orbitals(torch, n, k, seed):
    import numpy as np
    return torch.as_tensor(np.random.default_rng(seed).normal(size=(n, k)) / np.sqrt(n),
                           device='cuda')


def test_functional_potentials_are_energy_derivatives():
    """On the grid: d/dD of E_xc = sum_p W rho e_xc is the quadrature of
    v_xc, and d/dD_e, d/dD_n of E_epc = sum_p W rho_e e_epc are the
    quadratures of the two epc17-2 potentials (central differences along
    directions inside the occupied space, so that the density's change stays
    a bounded fraction of the density: rho^(4/3) is not smooth at zero)."""
    import torch
    from helpers import HCN
    from napmo_b200.scf import GridAPMO, epc17_2_device, lda_xc
    from napmo_b200.system import build_system
    ap = GridAPMO(build_system(HCN, 'CC-PVDZ', quantum=(0,)), 'H_1', 50, 110, exchange='lda',
                  correlation='epc17-2')
    e, n, W = ap.e, ap.nuc, ap.W
    Ce, Cn = _orbitals(torch, e.n, 7, 1), _orbitals(torch, n.n, 1, 2)
    De, Dn = 2.0 * Ce @ Ce.T, Cn @ Cn.T
    Cr = Ce @ (0.03 * _orbitals(torch, 7, 3, 3) * 7 ** 0.5)
    de, dn = Cr @ Cr.T, 1e-2 * Dn
    eps = 1e-2

    def exc(D):
        rho = e.fb.density(D)
        return float((W * rho * lda_xc(torch, rho)[1]).sum())

    def epc(D1, D2):
        r1, r2 = e.fb.density(D1), n.fb.density(D2)
        return float((W * r1 * epc17_2_device(torch, r1, r2)[0]).sum())

    rho_e, rho_n = e.fb.density(De), n.fb.density(Dn)
    vxc = lda_xc(torch, rho_e)[0]
    _, pe, pn = epc17_2_device(torch, rho_e, rho_n)
    checks = [
        ((exc(De + eps * de) - exc(De - eps * de)) / (2 * eps),
         float((e.fb.quadrature(0.0, None, vext=vxc) * de).sum())),
        ((epc(De + eps * de, Dn) - epc(De - eps * de, Dn)) / (2 * eps),
         float((e.fb.quadrature(0.0, None, vext=pe) * de).sum())),
        ((epc(De, Dn + eps * dn) - epc(De, Dn - eps * dn)) / (2 * eps),
         float((n.fb.quadrature(0.0, None, vext=pn) * dn).sum())),
    ]
    for fd, an in checks:
        assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)
