"""ORACLE -- test infrastructure only.

Geometries of the measured workloads for the host (reference) arm of
bench.py, written without the napmo_b200 package so that the reference
process never loads libnapmo.so.  The same constructions as
napmo_b200/system.py (checked equal, bit for bit, by tests/test_scf_oracle.py).
"""
import math

import numpy as np

H2O = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.757, 0.587)), ('H', (0.0, -0.757, 0.587))]
HCN = [('H', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 1.066)), ('N', (0.0, 0.0, 2.222))]


def alkane_geometry(ncarbon=20, cc=1.54, ch=1.09):
    """All-trans alkane CnH2n+2 (angstrom): carbons on a planar zig-zag with
    tetrahedral angles, two H per carbon out of the backbone plane, one more
    H on each end where the next carbon would sit."""
    theta = math.acos(-1.0 / 3.0)
    half = theta / 2.0
    dz = cc * math.sin(half)
    dy = cc * math.cos(half)
    carbons = [np.array([0.0, (dy / 2.0) * (1 if i % 2 == 0 else -1), i * dz])
               for i in range(ncarbon)]
    atoms = [('C', tuple(c)) for c in carbons]
    hx = ch * math.sin(half)
    for i, c in enumerate(carbons):
        side = 1.0 if i % 2 == 0 else -1.0
        hy = ch * math.cos(half) * side
        atoms.append(('H', (hx, c[1] + hy, c[2])))
        atoms.append(('H', (-hx, c[1] + hy, c[2])))
    for end, virt in ((0, -1), (ncarbon - 1, ncarbon)):
        c = carbons[end]
        nxt = np.array([0.0, (dy / 2.0) * (1 if virt % 2 == 0 else -1), virt * dz])
        d = (nxt - c) / np.linalg.norm(nxt - c)
        atoms.append(('H', tuple(c + ch * d)))
    return atoms
