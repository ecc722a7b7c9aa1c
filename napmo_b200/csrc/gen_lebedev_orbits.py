"""Generate ``lebedev_orbits.inc``: the octahedral-orbit parameters of the
Lebedev-Laikov spherical quadratures (V. I. Lebedev, D. N. Laikov, Doklady
Mathematics 59, 477 (1999)).

Each rule of order N is a list of symmetry orbits ``(code, a, b, v)``; code 1..6
names the orbit type (6, 12, 8, 24, 24 or 48 points), ``a``/``b`` are the free
coordinates of the generating point and ``v`` the weight of every point of the
orbit.  The numbers are published constants; grid points must match the ones
nAPMO builds bit for bit, so they are read from the rule tables nAPMO ships
(``src/grid/sphere_lebedev_rule.cpp``) and re-emitted with ``repr`` (shortest
round-trip decimal, so the C compiler parses the identical double).  The point
expansion of each orbit is done by ``lebedev.cpp`` in this package.

Usage: python gen_lebedev_orbits.py <path to sphere_lebedev_rule.cpp>
"""
import re
import sys
import os

ORDERS = [6, 14, 26, 38, 50, 74, 86, 110, 146, 170, 194, 230, 266, 302, 350,
          434, 590, 770, 974, 1202, 1454, 1730, 2030, 2354, 2702, 3074, 3470,
          3890, 4334, 4802, 5294, 5810]
ORBIT_SIZE = {1: 6, 2: 12, 3: 8, 4: 24, 5: 24, 6: 48}


def parse(src):
    rules = {}
    for order in ORDERS:
        m = re.search(r'void ld%04d\(double \*x, double \*y, double \*z, double \*w\)' % order, src)
        if m is None:
            raise RuntimeError('rule %d not found' % order)
        body = src[m.end():]
        body = body[:body.index('\n}')]
        a = b = 0.0
        v = None
        orbits = []
        for line in body.splitlines():
            line = line.strip()
            ma = re.match(r'^a = ([-+0-9.eE]+);', line)
            mb = re.match(r'^b = ([-+0-9.eE]+);', line)
            mv = re.match(r'^v = ([-+0-9.eE]+);', line)
            mg = re.match(r'^n = n \+ gen_oh\((\d), a, b, v', line)
            if ma:
                a = float(ma.group(1))
            elif mb:
                b = float(mb.group(1))
            elif mv:
                v = float(mv.group(1))
            elif mg:
                orbits.append((int(mg.group(1)), a, b, v))
        if sum(ORBIT_SIZE[o[0]] for o in orbits) != order:
            raise RuntimeError('rule %d: orbit sizes do not add up' % order)
        rules[order] = orbits
    return rules


def emit(rules, path):
    with open(path, 'w') as f:
        f.write('/* Generated by gen_lebedev_orbits.py -- do not edit.\n'
                '   Lebedev-Laikov octahedral orbits: {rule order, orbit code, a, b, weight}. */\n')
        f.write('static const LebedevOrbit kLebedevOrbits[] = {\n')
        for order in ORDERS:
            for code, a, b, v in rules[order]:
                f.write('  {%d, %d, %r, %r, %r},\n' % (order, code, a, b, v))
        f.write('};\n')


if __name__ == '__main__':
    src_path = sys.argv[1]
    with open(src_path) as fh:
        rules = parse(fh.read())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'lebedev_orbits.inc')
    emit(rules, out)
    print('wrote', out, sum(len(v) for v in rules.values()), 'orbits')
