"""Record the ctypes bindings nAPMO declares for libnapmo into
tests/golden/napmo_bindings.json.

nAPMO's napmo/__init__.py sets `cext.<symbol>.argtypes = [...]` and
`cext.<symbol>.restype = ...` for every C symbol its Python layer calls.  The
file is read as text and parsed with `ast` (it is not imported: importing it
needs pylibxc and a built libnapmo).  The fixture lets the CPU tests check
this library's declarations and exports against nAPMO's bindings without the
nAPMO tree at test time.

Usage: python tests/golden/make_bindings.py /path/to/nAPMO (or NAPMO_REFERENCE set)
"""
import ast
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def bindings(init_py):
    with open(init_py) as f:
        tree = ast.parse(f.read())
    out = {}
    for node in ast.walk(tree):
        if not isinstance(node, ast.Assign) or len(node.targets) != 1:
            continue
        t = node.targets[0]
        if not (isinstance(t, ast.Attribute) and t.attr in ('argtypes', 'restype')
                and isinstance(t.value, ast.Attribute)
                and isinstance(t.value.value, ast.Name) and t.value.value.id == 'cext'):
            continue
        name = t.value.attr
        entry = out.setdefault(name, {'line': node.lineno})
        if t.attr == 'argtypes':
            if not isinstance(node.value, ast.List):
                raise ValueError('%s: argtypes is not a list literal' % name)
            entry['argtypes'] = [ast.unparse(e) for e in node.value.elts]
        else:
            entry['restype'] = ast.unparse(node.value)
        entry['line'] = min(entry['line'], node.lineno)
    return out


def main(ref):
    b = bindings(os.path.join(ref, 'napmo', '__init__.py'))
    with open(os.path.join(HERE, 'napmo_bindings.json'), 'w') as f:
        json.dump({'source': 'napmo/__init__.py', 'bindings': b}, f, indent=1, sort_keys=True)
    print('recorded %d bindings' % len(b))


if __name__ == '__main__':
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('NAPMO_REFERENCE')
    if not ref:
        sys.exit('usage: make_bindings.py <nAPMO source tree> (or set NAPMO_REFERENCE)')
    main(ref)
