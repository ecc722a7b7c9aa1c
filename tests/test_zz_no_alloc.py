"""napmo_gpu_quadrature_noalloc: the quadrature for callers that cannot
allocate device memory while calling the library (hosts that budget all GPU
memory themselves, callers that must not let an allocation synchronise the
device).  Its split-K scratch is a fixed 16 MiB array inside libnapmo.so.

Checked through the C-ABI against napmo_gpu_quadrature (the allocating entry
point) on two calls in a row, within the quadrature tolerance of the parity
tests (1e-10 of max|F|); the two allocation-free calls must agree bit for bit
with each other.  The exact size boundary is pinned: n = 1920 (one chunk
covers every point) is accepted and n = 1921 refused.  At the H2O size the
result is also compared with the oracle's quadrature, and an empty grid
gives F = 0.  This
file is collected last so that a run stopping at the first failure has run
every other test already; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]


def _lib():
    from napmo_b200 import cext
    f = cext.lib.napmo_gpu_quadrature_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return cext


@pytest.mark.parametrize('n,npoint', [(25, 16500), (300, 40000), (1920, 3000)])
def test_noalloc_matches_allocating_quadrature(n, npoint):
    import torch
    cext = _lib()
    rng = np.random.default_rng(n)
    ld = (npoint + 127) // 128 * 128
    phi = np.zeros((n, ld))
    phi[:, :npoint] = rng.normal(size=(n, npoint)) * np.exp(-rng.uniform(0, 4, size=(n, 1)))
    wv = np.zeros(ld)
    wv[:npoint] = rng.uniform(-1.0, 1.0, size=npoint) * 1e-3
    dphi = torch.as_tensor(phi, device='cuda')
    dwv = torch.as_tensor(wv, device='cuda')
    stream = torch.cuda.current_stream().cuda_stream
    F_ref = torch.empty((n, n), dtype=torch.float64, device='cuda')
    cext.checked(cext.lib.napmo_gpu_quadrature(n, npoint, dphi.data_ptr(), None, ld,
                                               dwv.data_ptr(), F_ref.data_ptr(), stream))
    outs = []
    for _ in range(2):
        F = torch.full((n, n), float('nan'), dtype=torch.float64, device='cuda')
        cext.checked(cext.lib.napmo_gpu_quadrature_noalloc(n, npoint, dphi.data_ptr(), None, ld,
                                                           dwv.data_ptr(), F.data_ptr(), stream))
        torch.cuda.synchronize()
        outs.append(F.cpu().numpy())
    ref = F_ref.cpu().numpy()
    scale = np.abs(ref).max()
    for F in outs:
        assert np.all(np.isfinite(F))
        assert np.abs(F - ref).max() <= 1e-10 * scale
        assert np.array_equal(F, F.T)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_matches_the_oracle(oracle):
    import torch
    cext = _lib()
    n, npoint = 25, 16500
    rng = np.random.default_rng(7)
    ld = (npoint + 127) // 128 * 128
    phi = np.zeros((n, ld))
    phi[:, :npoint] = rng.normal(size=(n, npoint))
    wv = np.zeros(ld)
    wv[:npoint] = rng.uniform(-1.0, 1.0, size=npoint) * 1e-3
    dphi = torch.as_tensor(phi, device='cuda')
    dwv = torch.as_tensor(wv, device='cuda')
    F = torch.empty((n, n), dtype=torch.float64, device='cuda')
    cext.checked(cext.lib.napmo_gpu_quadrature_noalloc(n, npoint, dphi.data_ptr(), None, ld,
                                                       dwv.data_ptr(), F.data_ptr(),
                                                       torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    ones = np.ones(npoint)
    ref = oracle.quadrature(phi[:, :npoint].copy(), wv[:npoint].copy(), ones, ones)
    assert np.abs(F.cpu().numpy() - ref).max() <= 1e-10 * np.abs(ref).max()


def test_noalloc_empty_grid_gives_zero():
    import torch
    cext = _lib()
    n = 40
    dphi = torch.zeros((n, 128), dtype=torch.float64, device='cuda')
    dwv = torch.zeros(128, dtype=torch.float64, device='cuda')
    F = torch.full((n, n), float('nan'), dtype=torch.float64, device='cuda')
    stream = torch.cuda.current_stream().cuda_stream
    cext.checked(cext.lib.napmo_gpu_quadrature_noalloc(n, 0, dphi.data_ptr(), None, 128,
                                                       dwv.data_ptr(), F.data_ptr(), stream))
    torch.cuda.synchronize()
    assert np.array_equal(F.cpu().numpy(), np.zeros((n, n)))


@pytest.mark.parametrize('n', [1921, 2000])
def test_noalloc_rejects_sizes_beyond_the_fixed_scratch(n):
    import torch
    cext = _lib()
    npoint = 128
    ld = 128
    dphi = torch.zeros((n, ld), dtype=torch.float64, device='cuda')
    dwv = torch.zeros(ld, dtype=torch.float64, device='cuda')
    F = torch.zeros((n, n), dtype=torch.float64, device='cuda')
    st = cext.lib.napmo_gpu_quadrature_noalloc(n, npoint, dphi.data_ptr(), None, ld,
                                               dwv.data_ptr(), F.data_ptr(),
                                               torch.cuda.current_stream().cuda_stream)
    assert st != 0
    code, msg = cext.last_error()
    assert '1920' in msg
