"""Regenerate the data tables of this package from nAPMO's data directory.

* ``elements.json``: per element symbol the atomic number, mass and the
  Bragg-Slater-type radii (``atomic_radii``, ``atomic_radii_2``) nAPMO uses
  for the Chebyshev radial grids (napmo/grids/radial.py:20-48).
* ``basis.json``: the Gaussian basis sets (published data from the EMSL Basis
  Set Exchange, deMon2k format in nAPMO) that the tests and the benchmark
  use, as ``{basis: {particle: [[l, [exponents], [coefficients]], ...]}}``
  in file order, which fixes the function order.

Usage: python gen_data.py <nAPMO data dir>   (e.g. .../napmo/data)
"""
import json
import os
import re
import sys

BASES = ['CC-PVDZ', 'STO-3G', '6-311G', 'DZSNB']


def parse_basis(text):
    text = re.sub('#.*\n?', '', text)
    text = re.sub(r'(?imu)^\s*\n', '', text)
    lines = text.splitlines()
    out = {}
    i = 0
    while i < len(lines):
        m = re.match(r'^O-\S*\s+(\S+)', lines[i].strip())
        if not m:
            i += 1
            continue
        particle = m.group(1)
        ncont = int(lines[i + 1].strip())
        k = i + 2
        conts = []
        for _ in range(ncont):
            head = lines[k].split()
            l, nprim = int(head[1]), int(head[2])
            k += 1
            exps, coefs = [], []
            for _ in range(nprim):
                a, c = lines[k].split()[:2]
                exps.append(float(a))
                coefs.append(float(c))
                k += 1
            conts.append([l, exps, coefs])
        out.setdefault(particle, conts)
        i = k
    return out


def main(datadir):
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(datadir, 'atomic_elements.json')) as f:
        el = json.load(f)
    keep = {}
    for sym, rec in el.items():
        keep[sym] = {k: rec.get(k) for k in
                     ('atomic_number', 'mass', 'atomic_radii', 'atomic_radii_2')}
    with open(os.path.join(here, 'elements.json'), 'w') as f:
        json.dump(keep, f, indent=0, sort_keys=True)
    bases = {}
    for name in BASES:
        with open(os.path.join(datadir, 'basis', name)) as f:
            bases[name] = parse_basis(f.read())
    with open(os.path.join(here, 'basis.json'), 'w') as f:
        json.dump(bases, f, separators=(',', ':'))
    print('elements:', len(keep), 'bases:', {k: len(v) for k, v in bases.items()})


if __name__ == '__main__':
    main(sys.argv[1])
