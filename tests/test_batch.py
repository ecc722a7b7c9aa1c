"""Batched workload generator (host side; the batched builds are GPU tests)."""
import numpy as np


def test_random_batch_is_seeded_and_in_range():
    from napmo_b200.system import ANGULAR_SIZES, random_batch
    a = random_batch(nmol=12, seed=5)
    b = random_batch(nmol=12, seed=5)
    assert a == b
    assert random_batch(nmol=12, seed=6) != a
    for m in a:
        na = len(m['atoms'])
        assert 3 <= na <= 30
        assert len(m['nrad']) == na and len(m['nang']) == na
        assert all(50 <= r <= 100 for r in m['nrad'])
        assert all(g in ANGULAR_SIZES for g in m['nang'])
        xyz = np.array([p for _, p in m['atoms']])
        bonds = np.linalg.norm(np.diff(xyz, axis=0), axis=1)
        assert np.all((bonds >= 1.0 - 1e-12) & (bonds <= 1.5 + 1e-12))
        d = np.linalg.norm(xyz[:, None] - xyz[None], axis=2)
        assert d[np.triu_indices(na, 1)].min() >= 1.0 - 1e-12
        assert all(s in 'HCNO' for s, _ in m['atoms'])
