"""Local functionals on the GPU (napmo_gpu_lda_xc, napmo_gpu_epc17_2) against
nAPMO's LDA fixtures and the CPU restatement (oracle/xc.py).  The device
math (cbrt, log, atan) may differ from the host's in the last bits, hence
tolerances of a few ulps of the largest value."""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'xc_lda.npz')


def test_lda_matches_napmo_fixtures():
    import napmo_b200 as nb
    g = np.load(GOLDEN)
    f = nb.Functional('e-')
    zc, vc = f.compute_correlation(g['rho'])
    zx, vx = f.compute_exchange(g['rho'])
    assert zc.shape == (g['rho'].size, 1)
    for got, ref in ((zx, g['x_zk']), (vx, g['x_vrho']), (zc, g['c_zk']), (vc, g['c_vrho'])):
        assert np.abs(got[:, 0] - ref).max() <= 1e-14 * np.abs(ref).max()
    assert np.all(zx[g['rho'] < 1e-24] == 0.0) and np.all(vc[g['rho'] < 1e-24] == 0.0)


def test_lda_device_tensors_match_oracle():
    import torch
    import napmo_b200 as nb
    import xc
    rho = np.geomspace(1e-30, 1e3, 100000)
    f = nb.Functional('e-')
    zx, vx = f.compute_exchange(torch.as_tensor(rho, device='cuda'))
    assert zx.is_cuda
    rx, rvx = xc.lda_x(rho)
    rc, rvc = xc.lda_c_vwn(rho)
    zc, vc = f.compute_correlation(rho)
    assert np.abs(zx.cpu().numpy()[:, 0] - rx).max() <= 1e-14 * np.abs(rx).max()
    assert np.abs(vx.cpu().numpy()[:, 0] - rvx).max() <= 1e-14 * np.abs(rvx).max()
    assert np.abs(zc[:, 0] - rc).max() <= 1e-14 * np.abs(rc).max()
    assert np.abs(vc[:, 0] - rvc).max() <= 1e-14 * np.abs(rvc).max()


@pytest.mark.parametrize('tiny', [False, True])
def test_epc17_2_matches_oracle(tiny):
    import napmo_b200 as nb
    import xc
    rng = np.random.default_rng(7)
    e = rng.random(70001) * 3 + 1e-6
    n = rng.random(70001) * 40 + 1e-6
    if tiny:
        n[12345] = 0.0                 # switches every point to the alternative potentials
    ref = xc.epc17_2(e, n)
    got = nb.epc17_2(e, n)
    for a, b in zip(got, ref):
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    f = nb.isc_functional_selector('epc17-2')
    assert f is nb.epc17_2 and nb.isc_functional_selector(None) is None
    with pytest.raises(NotImplementedError):
        nb.isc_functional_selector('epc17-1')
