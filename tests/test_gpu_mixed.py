"""Int8-slice tensor-core contractions (tcgen05 kind::i8) on the GPU.

Two checks per result: (1) the kernels compute exactly the scheme restated in
oracle/ozaki.py (the same screened points; integer parts exact; only the
order of the final FP64 sums differs, so agreement to 1e-12 relative), and
(2) the scheme's distance from the FP64 path: rho within 1e-7 of max|rho| at
the kept points (and wb w rho negligible at the others), F within 1e-8 of
max|F|, and the Fock-build energy 1/2 tr(D F) within 1e-6 Eh.
"""
import numpy as np
import pytest

from conftest import gpu_available
from helpers import H2O, product_system, random_density

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]

BUTANE = [('C', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 1.54)), ('C', (0.0, 1.45, 2.05)),
          ('C', (0.0, 1.45, 3.59)), ('H', (1.03, 0.0, -0.36)), ('H', (-1.03, 0.0, -0.36)),
          ('H', (0.0, -1.03, -0.36)), ('H', (1.03, -0.5, 1.9)), ('H', (-1.03, -0.5, 1.9)),
          ('H', (1.03, 1.95, 1.7)), ('H', (-1.03, 1.95, 1.7)), ('H', (1.03, 0.95, 3.95)),
          ('H', (-1.03, 0.95, 3.95)), ('H', (0.0, 2.48, 3.95))]


def _phi_host(fb):
    return fb.phi().cpu().numpy()[:, :fb.npoint].copy()


def _screened_scheme(tc, phi, grid):
    """Kept points of the int8 plan, checked against the oracle's screen."""
    import ozaki
    keep = tc.kept_points().cpu().numpy()
    assert np.array_equal(keep, ozaki.screen(phi, grid.becke_weights, grid.weights))
    assert 0 < keep.sum() <= keep.size
    return keep


def _scheme_density(phi, D, keep):
    import ozaki
    rs = np.zeros(phi.shape[1])
    rs[keep] = ozaki.density(phi[:, keep], D)
    return rs


def _scheme_quadrature(phi, wv, wb, w, keep):
    import ozaki
    return ozaki.quadrature(phi[:, keep], wv[keep], wb[keep], w[keep])


@pytest.mark.parametrize('atoms,nrad,nang', [(H2O, 50, 110), (BUTANE, 40, 110)])
def test_int8_matches_scheme_and_fp64(atoms, nrad, nang):
    import napmo_b200 as nb
    import ozaki
    ms, grid = product_system(atoms, nrad=nrad, nang=nang)
    basis = ms['e-']['basis']
    n = basis['nbasis']
    D = random_density(n, ms['e-']['occupation'])
    rng = np.random.default_rng(7)
    v = 1.0 + rng.random(grid.size)
    f64 = nb.FockBuilder(grid, basis, -1)
    tc = nb.FockBuilder(grid, basis, -1, precision='int8x4')
    phi = _phi_host(f64)
    wb, w = grid.becke_weights, grid.weights
    keep = _screened_scheme(tc, phi, grid)
    assert f64.kept_points() is None
    r64 = f64.density(D).cpu().numpy()
    r8 = tc.density(D).cpu().numpy()
    assert tc.tc_status() == 0
    rs = _scheme_density(phi, D, keep)
    assert np.abs(r8 - rs).max() <= 1e-12 * np.abs(rs).max()
    assert np.abs(r8 - r64)[keep].max() <= 1e-7 * np.abs(r64).max()
    assert np.all(r8[~keep] == 0.0)
    # |rho(p)| <= sum |D| max phi^2 and |wb w| max phi^2 < 1e-24 at a dropped point
    assert np.abs(wb * w * r64)[~keep].sum() <= (~keep).sum() * 1e-24 * np.abs(D).sum()

    F64 = f64.quadrature(1.0, v).cpu().numpy()
    F8 = tc.quadrature(1.0, v).cpu().numpy()
    assert tc.tc_status() == 0
    assert np.array_equal(F8, F8.T)
    Fs = _scheme_quadrature(phi, (wb * w) * v, wb, w, keep)
    assert np.abs(F8 - Fs).max() <= 1e-12 * np.abs(Fs).max()
    assert np.abs(F8 - F64).max() <= 1e-8 * np.abs(F64).max()
    # determinism: same bits on a second call
    assert np.array_equal(F8, tc.quadrature(1.0, v).cpu().numpy())
    assert np.array_equal(r8, tc.density(D).cpu().numpy())


def test_int8_uneven_grid_and_signed_potential():
    """Per-atom grid sizes differ, the potential changes sign, n is not a
    multiple of any tile."""
    import napmo_b200 as nb
    import ozaki
    from napmo_b200.system import build_system
    ms = build_system(H2O, 'CC-PVDZ')
    grid = nb.BeckeGrid(ms['e-'], [40, 30, 30], [110, 50, 86])
    basis = ms['e-']['basis']
    rng = np.random.default_rng(11)
    v = rng.normal(size=grid.size)
    tc = nb.FockBuilder(grid, basis, -1, precision='int8x4')
    f64 = nb.FockBuilder(grid, basis, -1)
    F8 = tc.quadrature(1.0, v).cpu().numpy()
    F64 = f64.quadrature(1.0, v).cpu().numpy()
    wb, w = grid.becke_weights, grid.weights
    phi = _phi_host(f64)
    keep = _screened_scheme(tc, phi, grid)
    Fs = _scheme_quadrature(phi, (wb * w) * v, wb, w, keep)
    assert tc.tc_status() == 0
    assert np.abs(F8 - Fs).max() <= 1e-12 * np.abs(Fs).max()
    assert np.abs(F8 - F64).max() <= 1e-8 * np.abs(F64).max()


@pytest.mark.parametrize('atoms,nrad,nang,nocc', [(H2O, 50, 110, 5), (BUTANE, 40, 110, 17)])
def test_int8_fock_build_energy(atoms, nrad, nang, nocc):
    import napmo_b200 as nb
    ms, grid = product_system(atoms, nrad=nrad, nang=nang)
    basis = ms['e-']['basis']
    D = random_density(basis['nbasis'], nocc)
    F64, rho64, _ = nb.FockBuilder(grid, basis, 8).build(D)
    tc = nb.FockBuilder(grid, basis, 8, precision='int8x4')
    F8, rho8, _ = tc.build(D)
    assert tc.tc_status() == 0
    E64 = 0.5 * float((F64.cpu().numpy() * D).sum())
    E8 = 0.5 * float((F8.cpu().numpy() * D).sum())
    assert abs(E64 - E8) <= 1e-6
    n64 = grid.integrate(rho64.cpu().numpy())
    n8 = grid.integrate(rho8.cpu().numpy())
    assert abs(n64 - n8) <= 1e-7


def test_bounded_wait_times_out_and_reports():
    """The tensor-core kernels' mbarrier waits are bounded: a wait on a barrier
    that nothing arrives on gives up (about 2 s), records error 5 for
    napmo_tc_status, and a second role waiting elsewhere leaves through the
    abort flag; the context stays usable."""
    import torch
    from napmo_b200 import cext
    stream = torch.cuda.current_stream().cuda_stream
    assert cext.lib.napmo_tc_status(stream, 1) in (0, 5)
    cext.lib.napmo_tc_status(stream, 1)
    out = torch.full((2,), 7, dtype=torch.int32, device='cuda')
    cext.checked(cext.lib.napmo_tc_wait_selftest(out.data_ptr(), stream))
    torch.cuda.synchronize()
    assert out.cpu().tolist() == [0, 0]
    assert cext.lib.napmo_tc_status(stream, 1) == 5
    assert cext.lib.napmo_tc_status(stream, 1) == 0
    x = torch.ones(1024, device='cuda', dtype=torch.float64)
    assert float(x.sum()) == 1024.0


def test_release_fp64_phi():
    """'int8x4' plans may free their FP64 phi: the int8 builds give the same
    bits without it, the device gets its n x ld doubles back, and whatever
    needs phi again (phi(), a switch back to FP64) evaluates it to the same
    bits."""
    import torch
    import napmo_b200 as nb
    ms, grid = product_system(BUTANE, nrad=40, nang=110)
    basis = ms['e-']['basis']
    D = random_density(basis['nbasis'], 17)
    tc = nb.FockBuilder(grid, basis, 8, precision='int8x4')
    phi0 = tc.phi().cpu().numpy().copy()
    tc.set_precision('fp64')
    F64, rho64, _ = tc.build(D)
    F64, rho64 = F64.cpu().numpy(), rho64.cpu().numpy()
    tc.set_precision('int8x4')
    F8, rho8, _ = tc.build(D)
    F8, rho8 = F8.cpu().numpy(), rho8.cpu().numpy()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    tc.release_fp64_phi()
    freed = torch.cuda.mem_get_info()[0] - free0
    assert freed >= 0.9 * tc.n * tc.ld * 8
    G8, s8, _ = tc.build(D)
    assert tc.tc_status() == 0
    assert np.array_equal(G8.cpu().numpy(), F8)
    assert np.array_equal(s8.cpu().numpy(), rho8)
    tc.release_fp64_phi()                      # twice is harmless
    assert np.array_equal(tc.phi().cpu().numpy(), phi0)
    tc.release_fp64_phi()
    tc.set_precision('fp64')
    G64, s64, _ = tc.build(D)
    assert np.array_equal(G64.cpu().numpy(), F64)
    assert np.array_equal(s64.cpu().numpy(), rho64)
    with pytest.raises(nb.cext.NapmoError):
        tc.release_fp64_phi()                  # FP64 builds read phi
