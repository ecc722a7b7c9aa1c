"""Batched Fock builds (one CUDA-graph launch over molecules of uneven grid
and basis sizes) against per-molecule builds."""
import numpy as np
import pytest

from conftest import gpu_available
from helpers import random_density

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason='needs a CUDA device')]


def _molecules(nmol=6, seed=11):
    import napmo_b200 as nb
    from napmo_b200.system import build_system, random_batch
    mols = random_batch(nmol=nmol, seed=seed, natom=(3, 7), nrad=(20, 35),
                        angular=(50, 86, 110, 146))
    out = []
    for m in mols:
        ms = build_system(m['atoms'], 'CC-PVDZ')
        e = ms['e-']
        grid = nb.BeckeGrid(e, m['nrad'], m['nang'])
        out.append((e, grid))
    return out


def test_batch_equals_single_builds_fp64_and_int8():
    import torch
    import napmo_b200 as nb
    mols = _molecules()
    builders = [nb.FockBuilder(g, e['basis'], 'per-atom') for e, g in mols]
    Ds = [random_density(b.n, max(1, e['occupation']), seed=100 + i)
          for i, ((e, g), b) in enumerate(zip(mols, builders))]
    ref64 = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
    batch = nb.FockBatch(builders)
    Fs = [F.cpu().numpy() for F in batch.build(Ds)]
    torch.cuda.synchronize()
    for F, R in zip(Fs, ref64):
        assert np.array_equal(F, R)            # same kernels, same launch shapes
    # a second launch of the captured graph gives the same bits
    Fs2 = [F.cpu().numpy() for F in batch.build()]
    assert all(np.array_equal(a, b) for a, b in zip(Fs, Fs2))

    for b in builders:
        b.set_precision('int8x4')
    ref8 = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
    batch8 = nb.FockBatch(builders)
    cfg = batch8.tune(reps=2)
    assert cfg['nstream'] >= 1 and cfg['budget'] >= 1 and cfg['ms'] > 0
    F8 = [F.cpu().numpy() for F in batch8.build(Ds)]
    assert builders[0].tc_status() == 0
    for F, R, R64, D in zip(F8, ref8, ref64, Ds):
        # the tuned split-K chunking only reorders FP64 partial sums
        assert np.abs(F - R).max() <= 1e-12 * np.abs(R).max()
        assert abs(0.5 * float((F * D).sum()) - 0.5 * float((R64 * D).sum())) <= 1e-6


def test_batch_recaptures_after_plans_change():
    """A captured batch holds the device state of its plans.  Moving one
    molecule (grid + basis + refresh) and switching another to int8 must make
    the next batch build run on the new state: equal to fresh single builds."""
    import torch
    import napmo_b200 as nb
    mols = _molecules(nmol=3, seed=21)
    builders = [nb.FockBuilder(g, e['basis'], 'per-atom') for e, g in mols]
    Ds = [random_density(b.n, max(1, e['occupation']), seed=200 + i)
          for i, ((e, g), b) in enumerate(zip(mols, builders))]
    batch = nb.FockBatch(builders)
    batch.build(Ds)
    torch.cuda.synchronize()
    # move molecule 0 by a rigid shift
    e0, g0 = mols[0]
    shift = np.array([0.31, -0.17, 0.23])
    org = e0['basis'].origins()
    centres = np.array([p['origin'] for p in e0['particles']], dtype=np.float64)
    g0.set_centers(centres + shift)
    e0['basis'].set_origins(org + shift)
    builders[0].refresh()
    builders[1].set_precision('int8x4')
    Fs = [F.cpu().numpy() for F in batch.build()]
    assert builders[1].tc_status() == 0
    for F, b, D in zip(Fs, builders, Ds):
        R = b.build(D)[0].cpu().numpy()
        assert np.abs(F - R).max() <= 1e-12 * np.abs(R).max()


def test_batch_at_the_batched_configuration_sizes():
    """Three molecules at the sizes of the 64-molecule batch's range: 30 and 24
    atoms with 100 radial points and 590- / 434-point rules on some atoms,
    per-atom lmax up to 20.  The int8 batch equals its single builds and stays
    within 1e-6 Eh of the FP64 builds."""
    import torch
    import napmo_b200 as nb
    from napmo_b200.system import build_system, random_chain
    rng = np.random.default_rng(2026)
    specs = [(30, [100] * 30, [590 if i % 3 == 0 else 302 for i in range(30)]),
             (24, [50 + 2 * i for i in range(24)], [434 if i % 4 == 0 else 146 for i in range(24)]),
             (3, [100, 90, 80], [590, 590, 110])]
    builders, Ds = [], []
    for k, (na, nr, ng) in enumerate(specs):
        e = build_system(random_chain(rng, na), 'CC-PVDZ')['e-']
        grid = nb.BeckeGrid(e, nr, ng)
        b = nb.FockBuilder(grid, e['basis'], 'per-atom')
        builders.append(b)
        Ds.append(random_density(b.n, max(1, e['occupation']), seed=300 + k))
    ref64 = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
    for b in builders:
        b.set_precision('int8x4')
    ref8 = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
    batch = nb.FockBatch(builders)
    batch.tune(reps=1)
    F8 = [F.cpu().numpy() for F in batch.build(Ds)]
    torch.cuda.synchronize()
    assert builders[0].tc_status() == 0
    for F, R, R64, D in zip(F8, ref8, ref64, Ds):
        assert np.abs(F - R).max() <= 1e-12 * np.abs(R).max()
        assert abs(0.5 * float((F * D).sum()) - 0.5 * float((R64 * D).sum())) <= 1e-6


def test_stage_batch_equals_single_builds():
    """'stages' mode: one launch per stage for the whole batch (persistent
    density and quadrature launches over device work queues, one Poisson plan
    over all grids) gives every molecule's own build bit for bit, with and
    without FP64 point screening."""
    import torch
    import napmo_b200 as nb
    mols = _molecules(nmol=7, seed=5)
    builders = [nb.FockBuilder(g, e['basis'], 'per-atom') for e, g in mols]
    Ds = [random_density(b.n, max(1, e['occupation']), seed=200 + i)
          for i, ((e, g), b) in enumerate(zip(mols, builders))]
    for screen in (0.0, 1e-24):
        for b in builders:
            b.set_fp64_screening(screen)
        ref = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
        batch = nb.FockBatch(builders)
        batch.set_mode('stages')
        Fs = [F.cpu().numpy() for F in batch.build(Ds)]
        torch.cuda.synchronize()
        assert batch.status() == 0
        for F, R in zip(Fs, ref):
            assert np.array_equal(F, R)
        Fs2 = [F.cpu().numpy() for F in batch.build()]
        assert all(np.array_equal(a, c) for a, c in zip(Fs, Fs2))
    for b in builders:
        b.set_fp64_screening(0.0)


def test_stage_batch_queue_wait_runs_out():
    """A work queue that is never posted: every CTA's wait gives up after the
    per-launch limit and the queue's error word reads 5; the batch then builds
    correctly (no trap, no hang)."""
    import torch
    import napmo_b200 as nb
    mols = _molecules(nmol=3, seed=9)
    builders = [nb.FockBuilder(g, e['basis'], 'per-atom') for e, g in mols]
    Ds = [random_density(b.n, max(1, e['occupation']), seed=50 + i)
          for i, ((e, g), b) in enumerate(zip(mols, builders))]
    ref = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
    batch = nb.FockBatch(builders)
    batch.set_mode('stages')
    batch.build(Ds)
    assert batch.queue_selftest(0.2) == 5
    assert batch.status() == 0
    Fs = [F.cpu().numpy() for F in batch.build(Ds)]
    torch.cuda.synchronize()
    assert all(np.array_equal(F, R) for F, R in zip(Fs, ref))


def test_stage_batch_int8_equals_single_builds():
    """'stages' mode with int8 plans: every int8 stage (fold and slices of D,
    density, block scales, B images, quadrature, reduction) runs as one
    batched launch over all molecules, around one Poisson plan; each molecule's
    launch shape is its own plan's, so F equals its own int8 build bit for
    bit, also after tuning."""
    import torch
    import napmo_b200 as nb
    mols = _molecules(nmol=7, seed=5)
    builders = [nb.FockBuilder(g, e['basis'], 'per-atom', precision='int8x4') for e, g in mols]
    Ds = [random_density(b.n, max(1, e['occupation']), seed=200 + i)
          for i, ((e, g), b) in enumerate(zip(mols, builders))]
    ref = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
    batch = nb.FockBatch(builders)
    batch.set_mode('stages')
    Fs = [F.cpu().numpy() for F in batch.build(Ds)]
    torch.cuda.synchronize()
    assert builders[0].tc_status() == 0
    for F, R in zip(Fs, ref):
        assert np.array_equal(F, R)
    cfg = batch.tune(reps=2)
    assert cfg['ms'] > 0
    Fs = [F.cpu().numpy() for F in batch.build(Ds)]
    torch.cuda.synchronize()
    # the tuner left its budgets on the plans: their own builds use them too
    ref = [b.build(D)[0].cpu().numpy() for b, D in zip(builders, Ds)]
    for F, R in zip(Fs, ref):
        assert np.abs(F - R).max() <= 1e-12 * np.abs(R).max()
