"""Grid SCF of the electrons (napmo_b200.scf.GridRHF): convergence, electron
count, the closed-shell energy of H2O/cc-pVDZ with grid J and exchange, and
the int8 contractions against FP64 at the converged energy."""
import pytest

from conftest import gpu_available
from helpers import H2O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]


@pytest.mark.parametrize('exchange,lo,hi', [('hf', -76.035, -76.020), ('lda-x', -75.30, -75.10)])
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
