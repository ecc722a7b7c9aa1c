"""Build ``napmo_b200/lib/libnapmo.so`` in place for sm_100a.

Host translation units are compiled with g++ without -march and with
-ffp-contract=off, like nAPMO's own build (config.make: -O2 -fPIC), so grid
construction rounds exactly as the reference does.  CUDA units target
sm_100a only; becke.cu is compiled with --fmad=false (bit-exact Becke
weights).  Usage: python napmo_b200/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIBDIR = os.path.join(HERE, 'lib')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(LIBDIR, 'libnapmo.so')

NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
HOST_FLAGS = ['-O2', '-fPIC', '-std=c++17', '-ffp-contract=off', '-fno-fast-math']
CUDA_FLAGS = ARCH + ['-O3', '-lineinfo', '-std=c++17', '--expt-relaxed-constexpr',
                     '-Xcompiler', '-fPIC,-ffp-contract=off', '-Xptxas', '-warn-spills']
HOST_SOURCES = ['host.cpp']
CUDA_SOURCES = ['becke.cu', 'gto.cu', 'quad.cu', 'tc.cu', 'poisson.cu', 'capi_grid.cu',
                'capi_basis.cu', 'capi_quad.cu', 'capi_batch.cu', 'capi_scf.cu', 'grad.cu',
                'xc.cu', 'ints.cu']
EXTRA_CUDA = {'becke.cu': ['--fmad=false']}
LIBS = ['-lcusolver', '-lcublas']


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith(('.h', '.cuh', '.inc'))]


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = _headers()
    objs = []
    jobs = []
    for src in HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + '.o')
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(['g++'] + HOST_FLAGS + ['-c', s, '-o', o])
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + '.o')
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([NVCC] + CUDA_FLAGS + EXTRA_CUDA.get(src, []) + ['-c', s, '-o', o])
    procs = []
    for cmd in jobs:
        if verbose:
            print(' '.join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors='replace')
        if p.returncode != 0:
            failed = True
            sys.stderr.write('FAILED: %s\n%s\n' % (' '.join(cmd), text))
        elif verbose and text.strip():
            sys.stderr.write(text)
    if failed:
        raise RuntimeError('libnapmo build failed')
    if force or jobs or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ['-shared', '-o', LIB] + objs + LIBS
        if verbose:
            print(' '.join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)
