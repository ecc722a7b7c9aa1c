"""Shared builders: the same molecule as a napmo_b200 grid/basis and as an
oracle grid/basis description."""
import numpy as np

BOHR = 0.52917724924

H2O = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.757, 0.587)), ('H', (0.0, -0.757, 0.587))]
HCN = [('H', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 1.066)), ('N', (0.0, 0.0, 2.222))]


def product_system(atoms, basis='CC-PVDZ', nrad=50, nang=110, quantum=()):
    import napmo_b200 as nb
    from napmo_b200.system import build_system
    ms = build_system(atoms, basis, quantum=quantum)
    e = ms['e-']
    grid = nb.BeckeGrid(e, nrad, nang)
    return ms, grid


def oracle_system(oracle, library, elements, atoms, basis='CC-PVDZ', nrad=50, nang=110):
    centers = [np.array(xyz, dtype=np.float64) / BOHR for _, xyz in atoms]
    radii = [elements[s]['atomic_radii'] for s, _ in atoms]
    g = oracle.Grid(centers, radii, nrad, nang)
    fb = oracle.flat_basis(centers, [s for s, _ in atoms], library, basis)
    return g, fb


def random_density(n, nocc, seed=20261203):
    rng = np.random.default_rng(seed)
    C = rng.normal(size=(n, nocc)) / np.sqrt(n)
    return 2.0 * C @ C.T
