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


def test_polarised_lda_matches_oracle():
    """napmo_gpu_lda_xc_polarized against oracle/xc.py on random spin
    densities over 12 decades, with zeros, tiny totals and negative values;
    at zero spin it equals the unpolarised kernel."""
    import torch
    from napmo_b200 import cext
    import xc
    rng = np.random.default_rng(17)
    n = 5000
    ra = 10.0 ** rng.uniform(-10, 2, n)
    rb = 10.0 ** rng.uniform(-10, 2, n)
    ra[:20], rb[20:40] = 0.0, 0.0
    ra[40:50], rb[40:50] = 1e-26, 1e-26
    rb[50:60] = -1e-12
    a, b = torch.as_tensor(ra, device='cuda'), torch.as_tensor(rb, device='cuda')
    out = [torch.empty(n, dtype=torch.float64, device='cuda') for _ in range(6)]
    st = torch.cuda.current_stream().cuda_stream
    cext.checked(cext.lib.napmo_gpu_lda_xc_polarized(n, a.data_ptr(), b.data_ptr(),
                                                     *[o.data_ptr() for o in out], st))
    got = [o.cpu().numpy() for o in out]
    ref = list(xc.lda_x_polarized(ra, rb)) + list(xc.lda_c_vwn_polarized(ra, rb))
    for g_, r_ in zip(got, ref):
        assert np.abs(g_ - r_).max() <= 1e-14 * np.abs(r_).max()
    assert np.all(got[0][40:50] == 0.0) and np.all(got[3][40:50] == 0.0)
    # zero spin: the unpolarised kernel's values
    rho = torch.as_tensor(10.0 ** rng.uniform(-8, 2, n), device='cuda')
    h = (0.5 * rho).contiguous()
    pol = [torch.empty(n, dtype=torch.float64, device='cuda') for _ in range(6)]
    unp = [torch.empty(n, dtype=torch.float64, device='cuda') for _ in range(4)]
    cext.checked(cext.lib.napmo_gpu_lda_xc_polarized(n, h.data_ptr(), h.data_ptr(),
                                                     *[o.data_ptr() for o in pol], st))
    cext.checked(cext.lib.napmo_gpu_lda_xc(n, rho.data_ptr(), *[o.data_ptr() for o in unp], st))
    for p_, u_ in ((pol[0], unp[0]), (pol[1], unp[1]), (pol[3], unp[2]), (pol[4], unp[3])):
        assert float((p_ - u_).abs().max()) <= 1e-15 * float(u_.abs().max())
