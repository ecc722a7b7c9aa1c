"""Benchmark: grid Fock builds per second on one B200 (or N replicas).

Workload: linear alkane C20H42 (sp3, C-C 1.54 A, C-H 1.09 A), cc-pVDZ in
nAPMO's Cartesian form (510 functions), Becke grid of 100 Chebyshev radial x
302 Lebedev points per atom (62 atoms, 1,872,400 points), lmax = 14.  One
step = one grid Fock build of the electrons from a density matrix:
rho = diag(phi^T D phi), V_H by the Becke-Dickson Poisson solve, and
F = phi^T diag(w_becke w_quad V_H) phi -- the unit of work nAPMO repeats every
SCF iteration (psi_hybrid.py:81-110, ntwobody.py:15-46, nwavefunction.cpp).
D = 2 C C^T with C ~ N(0, 1/n) of shape n x 81 (seed 20261203); synthetic.
phi (7.6 GB) exceeds L2 (126 MB), so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'grid Fock builds/s (C20H42 cc-pVDZ, 100x302 Becke grid)'
UNIT = 'builds/s'
WORKLOAD = 'C20H42/cc-pVDZ Cartesian n=510, Becke 100x302 per atom, N=1872400, lmax=14'
SEED = 20261203
# DRAM bytes per (atom, point) pair of the potential evaluation kernel
# (profiles/poisson_kernels_C8H18_ncu.md: 122 MB read + 125 MB written for
# 26 atoms x 785,200 points); scaled by the pairs of the measured workload
EVAL_DRAM_BYTES_PER_PAIR = 297.079e9 * 2.051616e-3 / (26 * 785200)
TRAFFIC_SOURCE = ('ncu dram__bytes.sum.per_second x gpu__time_duration.sum of eval_pairs_kernel '
                  '(FP64 mode, first launch) at C8H18 100x302 (profiles/eval_pairs_C8H18_ncu.md): '
                  '0.61 GB for 20.4 M pairs, 29.9 B per (atom, point) pair (pair list, stored '
                  'u and 1/d, partial potential), scaled to this workload\'s pairs')


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=None,
                   help='timed steps (default 100 for c4, whose builds take 15 ms, else 10)')
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='napmo_b200')
    p.add_argument('--nrad', type=int, default=100)
    p.add_argument('--nang', type=int, default=302)
    p.add_argument('--ncarbon', type=int, default=20)
    p.add_argument('--cpu-points', type=int, default=4096)
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-scf', action='store_true', help='skip the SCF timing of the c4 line')
    p.add_argument('--workload', default='c4',
                   choices=['c4', 'c3', 'c5', 'c1', 'c2', 'c6', 'c7'],
                   help='c4: C20H42 single system (default); c3: batch of 64 random HCNO '
                        'chains with uneven per-atom grids, one CUDA-graph launch per batch')
    p.add_argument('--nmol', type=int, default=64)
    p.add_argument('--precision', default='auto', choices=['auto', 'fp64'],
                   help='auto: headline is the int8-slice tensor-core build when its energy '
                        'is within 1e-6 Eh of FP64 (checked in the same run), else FP64')
    args = p.parse_args()
    if args.steps is None:
        # c4 builds take 15 ms: 100 of them span the clock sampler's 100 ms
        # period many times; the reference arm's steps are 2 s CPU samples
        args.steps = 100 if args.workload == 'c4' and args.impl != 'reference' else 10
    return args


# ------------------------------------------------------------------ helpers
class ClockSampler(object):
    """nvidia-smi clocks and throttle reasons sampled every 100 ms.  start()
    returns once the first sample has arrived (nvidia-smi takes a moment to
    come up), so the timed region that follows is covered from its start."""
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.QUERY,
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        mhz, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.lines:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith('active'):
                    reasons.add(name)
        return {'sm_mhz': statistics.median(mhz) if mhz else None, 'sm_max_mhz': mx,
                'reasons': sorted(reasons), 'samples': len(mhz)}


def measured_peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), 'measured'
    return {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0}, 'fallback'


def fp64_gemm_peak(torch):
    """cuBLAS DGEMM 8192^3, best of 5 (FP64 denominator; the peaks file has none)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device='cuda')
    b = torch.randn(8192, 8192, dtype=torch.float64, device='cuda')
    best = 1e9
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2 * 8192 ** 3 / best / 1e12


def build_workload(args):
    import napmo_b200 as nb
    from napmo_b200.system import alkane_geometry, build_system
    atoms = alkane_geometry(args.ncarbon)
    ms = build_system(atoms, 'CC-PVDZ')
    e = ms['e-']
    grid = nb.BeckeGrid(e, args.nrad, args.nang)
    lmax = nb.lebedev_get_order(args.nang) // 2
    basis = e['basis']
    D = c4_density(basis['nbasis'], e['occupation'])
    return atoms, ms, grid, basis, lmax, D


def c4_config(world, n, N, lmax):
    """Workload description shared by the device arm and the host arm."""
    return {'workload': WORKLOAD, 'global_batch': world, 'n_basis': n, 'n_points': N,
            'lmax': lmax, 'parallelism': 'replicas' if world > 1 else 'single GPU',
            'l2': 'inputs larger than L2 (phi 7.6 GB)'}


# ------------------------------------------------------------- CPU baseline
def _ref_evaluation(r, centers, radii, nrad, lmax, y, dt, pts, v):
    """nAPMO's own multipole evaluation (horton/evaluate.cpp compiled from its
    sources into oracle/_ref, OpenMP as nAPMO builds it): per atom the lsize
    cubic splines of the decomposition on the atom's Chebyshev radial grid with
    nAPMO's potential extrapolation, evaluated at every sample point."""
    from ctypes import c_void_p
    for c, radius in zip(centers, radii):
        rt = r.ChebyshevRTransform_new(radius, nrad)
        splines, keep = [], []
        k = 0
        for l in range(lmax + 1):
            for _m in range(2 * l + 1):
                ext = r.PotentialExtrapolation_new(l)
                yy, dd = np.ascontiguousarray(y[k]), np.ascontiguousarray(dt[k])
                keep += [yy, dd]
                splines.append(r.CubicSpline_new(yy, dd, ext, rt, nrad))
                k += 1
        cell = r.Cell_new(None, 0)
        r.eval_decomposition_grid(np.array(splines, dtype=c_void_p), np.ascontiguousarray(c), v,
                                  pts, cell, len(splines), pts.shape[0])


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle as O
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'basis.json')) as f:
        lib = json.load(f)
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'elements.json')) as f:
        el = json.load(f)
    return O, lib, el


def c4_density(n, nocc):
    """D = 2 C C^T, C ~ N(0, 1/n) of shape n x nocc (seed 20261203)."""
    rng = np.random.default_rng(SEED)
    C = rng.normal(size=(n, nocc)) / np.sqrt(n)
    return 2.0 * C @ C.T


class HostWorkload(object):
    """The C20H42 build on the host, set up by the oracle alone (no
    libnapmo.so in the process): grid points and weights (atomic_grid.cpp),
    Becke weights of the sampled points and of two atoms' grids
    (becke.cpp:79-176 per point), the basis at the sampled points, the
    density of the two atoms' grids, and their Poisson splines
    (poisson_solver.py) as the spline coefficients of every atom of the same
    element."""

    def __init__(self, args):
        O, lib, el = _oracle()
        import workloads
        import scf as OS
        self.O = O
        atoms = workloads.alkane_geometry(args.ncarbon)
        self.syms = [s for s, _ in atoms]
        self.centers = [np.array(x) / 0.52917724924 for _, x in atoms]
        self.radii = [el[s]['atomic_radii'] for s in self.syms]
        self.grid = O.Grid(self.centers, self.radii, args.nrad, args.nang, becke=False)
        self.N = self.grid.size
        self.lmax = OS.lebedev_lmax(args.nang)
        self.nrad = args.nrad
        self.fb = O.flat_basis(self.centers, self.syms, lib, 'CC-PVDZ')
        self.n = self.fb['nf']
        nel = sum(el[s]['atomic_number'] for s in self.syms)
        self.D = c4_density(self.n, nel // 2)
        rng = np.random.default_rng(SEED)
        self.idx = np.sort(rng.choice(self.N, size=args.cpu_points, replace=False))
        self.pts = np.ascontiguousarray(self.grid.points[self.idx])
        self.bw = self.grid.becke_sample(self.idx)
        self.w = np.ascontiguousarray(self.grid.weights[self.idx])
        self.phi = np.ascontiguousarray(O.basis_compute(self.fb, self.pts).T)
        # one C and one H atom with their Becke weights in the molecule
        self.sub = [self.syms.index('C'), self.syms.index('H')]
        offs = self.grid.offsets
        sub_idx = np.concatenate([np.arange(offs[a], offs[a + 1]) for a in self.sub])

        class Sub(object):
            pass
        self.subgrid = Sub()
        self.subgrid.atoms = [self.grid.atoms[a] for a in self.sub]
        self.subgrid.becke = self.grid.becke_sample(sub_idx)
        phis = O.basis_compute(self.fb, self.grid.points[sub_idx])
        self.sub_rho = np.einsum('pi,pi->p', phis @ self.D, phis)
        del phis
        U = O.poisson_solver(self.subgrid, self.sub_rho, self.lmax)
        by_sym = {self.syms[a]: U[k] for k, a in enumerate(self.sub)}
        self.splines = [by_sym[s] for s in self.syms]


def cpu_baseline(args, hw):
    """nAPMO's path on the host cores, on a bounded sample of one build:
    density, multipole evaluation and quadrature on `cpu_points` grid points
    (scaled by N / sample), plus the projection and radial ODE solves of one
    C and one H atom (scaled by the atom counts).  Where nAPMO's own code runs
    here it is what is timed: the density by its numpy expression
    (psi_hybrid.py / psi_analytic.py: phi * D.dot(phi) per point, summed), the
    multipole evaluation by its compiled evaluate.cpp (oracle/_ref, when
    built), with the spline coefficients of the real density.  The quadrature
    is the oracle's streamed C restatement (nAPMO's materialises all orbital
    products, 1.95 TB here, and needs Eigen), and so are the projection and
    radial solves (scipy, as poisson_solver.py)."""
    O = hw.O
    N, D, phi = hw.N, hw.D, hw.phi
    t0 = time.perf_counter()
    Dgrid = np.array([p * D.dot(p) for p in phi.T]).T
    rho = Dgrid.sum(axis=0)
    t1 = time.perf_counter()
    v = np.zeros(args.cpu_points)
    lsize = (hw.lmax + 1) ** 2
    # nAPMO's library sets OpenMP's thread count from OMP_NUM_THREADS when it
    # loads (one thread if unset; utils/omp_helper.h): give it every core, as a
    # user of nAPMO would
    os.environ.setdefault('OMP_NUM_THREADS', str(os.cpu_count() or 1))
    r = O.ref_lib()
    t2 = time.perf_counter()
    for c, radius, (y, dt) in zip(hw.centers, hw.radii, hw.splines):
        if r is not None:
            _ref_evaluation(r, [c], [radius], hw.nrad, hw.lmax, y, dt, hw.pts, v)
        else:
            O.lib.orc_eval_decomposition(0, radius, 0.0, hw.nrad, lsize,
                                         np.ascontiguousarray(y), np.ascontiguousarray(dt),
                                         np.ascontiguousarray(c), args.cpu_points, hw.pts, v)
    t3 = time.perf_counter()
    F = O.quadrature(phi, v, hw.bw, hw.w)
    t4 = time.perf_counter()
    O.poisson_solver(hw.subgrid, hw.sub_rho, hw.lmax)
    t5 = time.perf_counter()
    del rho, F
    natom = len(hw.syms)
    scale = N / args.cpu_points
    parts = {'density': (t1 - t0) * scale, 'evaluation': (t3 - t2) * scale,
             'quadrature': (t4 - t3) * scale,
             'projection_radial': (t5 - t4) * natom / 2.0}
    t_build = sum(parts.values())
    return {'value': 1.0 / t_build, 'unit': UNIT, 'cores': O.threads(),
            'kind': 'reference' if r is not None else 'port',
            'sample': ('%d of %d points, scaled x%.0f: density by nAPMO\'s numpy expression, '
                       'multipole evaluation (%d atoms x %d splines of the real density, per '
                       'element) by %s, quadrature by the oracle\'s streamed C restatement '
                       '(OpenMP); projection + radial FEM solves (oracle, scipy spsolve) of 2 '
                       'of %d atoms, scaled x%.0f'
                       % (args.cpu_points, N, scale, natom, lsize,
                          "nAPMO's evaluate.cpp compiled from its sources (OpenMP, "
                          "OMP_NUM_THREADS = host cores)"
                          if r is not None else 'the oracle C restatement (OpenMP)',
                          natom, natom / 2.0)),
            'sample_seconds': t5 - t0, 'seconds_per_build': t_build,
            'seconds_per_part': parts}


# ------------------------------------------------- C1/C2: host SCF arms
# Iterations the oracle's SCFs take to converge (|dE| < 1e-9 Eh; the fixture
# tests/golden/scf_oracle.json records them): a timed iteration scaled by
# these is the host's time per SCF.
ORACLE_SCF_ITERATIONS = {'c1': 11, 'c2': 13}


def reference_scf(args, workload):
    """The oracle's grid SCF on the host cores (oracle/scf.py: nAPMO's
    arithmetic for the grid, the basis, the quadratures and the Poisson solves,
    the drivers' SCF loop).  C1: every step is one SCF iteration of H2O 50 x
    110 (J, orbital-pair exchange, DIIS, diagonalisation), continuing one SCF
    from the core guess.  C2 (HCN + quantum H, 100 x 302): every step is one
    iteration's Coulomb and coupling part (two densities, two Poisson solves,
    the quadratures of both species) plus the exchange of one of the seven
    occupied orbitals (n = 35 pair densities solved together), the exchange
    scaled by 7.  Value = seconds per iteration x the oracle SCF's
    iteration count."""
    O, lib, el = _oracle()
    import scf as OS
    import workloads
    niter = ORACLE_SCF_ITERATIONS[workload]
    times = []
    if workload == 'c1':
        orc = OS.GridRHF(workloads.H2O, lib, el, 50, 110)
        gen = orc.iterations(tol=1e-9)
        for _ in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            try:
                it, E, emax, conv, D = next(gen)
            except StopIteration:
                gen = orc.iterations(tol=1e-9)
                it, E, emax, conv, D = next(gen)
            times.append(time.perf_counter() - t0)
        sample = ('one SCF iteration per step (J by one Poisson solve, exchange by 5 x 25 '
                  'pair-density solves, DIIS, diagonalisation), x %d iterations' % niter)
        cfg = {'workload': 'C1: H2O cc-pVDZ (25 Cartesian functions), 50x110 per atom '
                           '(16,500 points), lmax 8, grid J and exchange, DIIS(6), 1e-8 Eh',
               'parallelism': 'single GPU'}
        metric = 'grid RHF SCF time, H2O / cc-pVDZ 50x110 (C1)'
        iter_s = times[args.warmup:]
    else:
        orc = OS.GridAPMO(workloads.HCN, lib, el, (0,), 100, 302)
        Ce, De, Cn, Dn = orc.guess()
        e, nuc, g = orc.e, orc.nuc, orc.grid
        qq = e.q * nuc.q
        iter_s = []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            rho_e, rho_n = O.density(e.phi, De), O.density(nuc.phi, Dn)
            V = OS.poisson_many(orc.plan, np.stack([rho_e, rho_n]))
            O.quadrature(e.phi, e.q * e.q * V[0] + qq * V[1], g.becke, g.weights)
            O.quadrature(nuc.phi, qq * V[0], g.becke, g.weights)
            t1 = time.perf_counter()
            psi = Ce[:, 0] @ e.phi
            Vk = OS.poisson_many(orc.plan, psi * e.phi)
            (e.phi * (orc.W * psi)) @ Vk.T
            t2 = time.perf_counter()
            if k >= args.warmup:
                iter_s.append((t1 - t0) + e.nocc * (t2 - t1))
        sample = ('per step one iteration\'s Coulomb + coupling part and the exchange of 1 '
                  'of 7 occupied orbitals (x7), x %d iterations' % niter)
        cfg = {'workload': 'C2: HCN, e- cc-pVDZ (35) + H nucleus 5s5p (20), 100x302 per '
                           'atom (90,600 points), lmax 14, DIIS(6), 1e-8 Eh',
               'parallelism': 'single GPU'}
        metric = 'grid APMO-RHF SCF time, HCN with quantum H, 100x302 (C2)'
    t_iter = statistics.median(iter_s)
    v = t_iter * niter
    cb = {'value': v, 'unit': 's per SCF', 'cores': O.threads(), 'kind': 'port',
          'sample': sample, 'seconds_per_iteration': t_iter}
    return {'impl': 'reference', 'metric': metric, 'value': v, 'unit': 's per SCF',
            'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': t_iter * 1e3, 'sample_scale_to_scf': niter,
            'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic', 'config': cfg, 'cpu_baseline': cb,
            'e2e': {'value': v, 'unit': 's per SCF', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}


# ------------------------------------------------------------ C3: batches
def run_batch(args, world, rank, dist=None):
    """64 seeded random {H,C,N,O} chains (3-30 atoms, bonds 1.0-1.5 A),
    cc-pVDZ, per-atom grids 50-100 x {110..590}, per-atom lmax from each
    atom's Lebedev rule; D = 2 C C^T of rank N_el/2.  One step = the Fock
    builds of all molecules in one CUDA-graph launch (FockBatch), FP64 and
    int8 (autotuned launch shape)."""
    import torch
    import napmo_b200 as nb
    from napmo_b200.parallel import max_over_ranks, shard_by_cost
    from napmo_b200.system import build_system, random_batch
    all_mols = random_batch(nmol=args.nmol, seed=SEED)
    # ranks share the batch by predicted cost (n^2 N), no data-path collective
    nb_of = {'H': 5, 'C': 15, 'N': 15, 'O': 15}
    costs = [float(sum(nb_of[s] for s, _ in m['atoms']) ** 2 *
                   sum(r * a for r, a in zip(m['nrad'], m['nang']))) for m in all_mols]
    mine = shard_by_cost(costs, world)[rank] if world > 1 else list(range(len(all_mols)))
    mols = [all_mols[i] for i in mine]
    builders, Ds, flops, npts = [], [], 0.0, 0
    t_setup = time.perf_counter()
    for i, m in zip(mine, mols):
        e = build_system(m['atoms'], 'CC-PVDZ')['e-']
        grid = nb.BeckeGrid(e, m['nrad'], m['nang'])
        fb = nb.FockBuilder(grid, e['basis'], 'per-atom')
        n = fb.n
        rng = np.random.default_rng(SEED + i)
        C = rng.normal(size=(n, max(1, e['occupation']))) / np.sqrt(n)
        Ds.append(2.0 * C @ C.T)
        builders.append(fb)
        flops += 4.0 * n * n * grid.size
        npts += grid.size
    t_setup = time.perf_counter() - t_setup
    stream = torch.cuda.current_stream()

    def timed(batch):
        batch.build(Ds)
        for _ in range(args.warmup):
            batch.build()
        torch.cuda.synchronize()
        sampler = ClockSampler(torch.cuda.current_device())
        sampler.start()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            batch.build()
        ev1.record(stream)
        ev1.synchronize()
        clk = sampler.stop()
        E = [0.5 * float((F * torch.as_tensor(D, device='cuda')).sum())
             for F, D in zip(batch._F, Ds)]
        t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3 / args.steps, dist, 'cuda')
        return t, clk, E

    # the tuner times builds of the batch's current densities: load them
    # first.  Both build modes of a batch are timed: 'streams' (the molecules'
    # own launch chains over capture streams, one graph) and 'stages' (one
    # launch per stage for the whole batch); the faster is reported.
    def best_mode():
        out = {}
        for mode in ('streams', 'stages'):
            bt = nb.FockBatch(builders)
            bt.set_mode(mode)
            bt.build(Ds)
            cfg = bt.tune(reps=2)
            t, clk, E = timed(bt)
            out[mode] = {'ms_per_batch': t * 1e3, 'tuned': cfg}
            if 'best' not in out or t < out['best'][0]:
                out['best'] = (t, clk, E, cfg, mode)
            del bt
        return out
    modes64 = best_mode()
    t64, clk64, E64, cfg64, mode64 = modes64.pop('best')
    for fb in builders:
        fb.set_precision('int8x4')
    modes8 = best_mode()
    t8, clk8, E8, cfg8, mode8 = modes8.pop('best')
    b8 = nb.FockBatch(builders)
    b8.set_mode(mode8)
    b8.build(Ds)
    b8.tune(reps=2)
    tc_err = builders[0].tc_status()
    dE = [abs(a - b) for a, b in zip(E8, E64)]
    dEmax = max_over_ranks(max(dE), dist, 'cuda')
    ok = max_over_ranks(tc_err, dist, 'cuda') == 0 and dEmax <= 1e-6
    headline = 'int8x4' if ok else 'fp64'
    t_dev = t8 if ok else t64
    bat = b8 if ok else None
    if not ok:
        for fb in builders:
            fb.set_precision('fp64')
        bat = nb.FockBatch(builders)
        bat.set_mode(mode64)
        bat.build(Ds)
        bat.tune(reps=2)
    # end to end: densities from pinned host memory in, every F read back
    hostD = [torch.as_tensor(D).pin_memory() for D in Ds]
    hostF = [torch.empty(D.shape, dtype=torch.float64).pin_memory() for D in Ds]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for dst, src in zip(bat._D, hostD):
            dst.copy_(src, non_blocking=True)
        bat.build()
        for dst, src in zip(hostF, bat._F):
            dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
    t_e2e = max_over_ranks((time.perf_counter() - t0) / args.steps, dist, 'cuda')
    nb_bytes = sum(8 * D.size for D in Ds)
    nmol = len(all_mols)
    line = {
        'metric': 'grid Fock builds/s, batch of %d random HCNO chains (C3)' % nmol,
        'value': nmol / t_dev, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': t_dev * 1e3, 'higher_is_better': True,
        'scaling': 'strong', 'vs_baseline': None, 'dtype': 'int8x4' if ok else 'f64',
        'data': 'synthetic',
        'config': {'workload': 'C3: %d random {H,C,N,O} chains of 3-30 atoms, cc-pVDZ, '
                               'per-atom 50-100 x {110..590} grids, per-atom lmax; molecules '
                               'shared by cost over the ranks' % nmol,
                   'n_points': npts, 'n_basis_range': [min(b.n for b in builders),
                                                       max(b.n for b in builders)],
                   'parallelism': 'one CUDA graph per batch (streams or stage launches)',
                   'l2': 'inputs larger than L2'},
        'e2e': {'value': nmol / t_e2e, 'unit': UNIT, 'h2d_bytes_per_step': nb_bytes,
                'd2h_bytes_per_step': nb_bytes},
        'gpu_launches': 1,
        'fp64': {'builds_per_s': nmol / t64, 'ms_per_batch': t64 * 1e3, 'tuned': cfg64,
                 'mode': mode64, 'modes': modes64},
        'mixed': {'builds_per_s': nmol / t8, 'ms_per_batch': t8 * 1e3, 'tuned': cfg8,
                  'mode': mode8, 'modes': modes8,
                  'speedup_vs_fp64': t64 / t8, 'tc_status': tc_err,
                  'energy_error_eh_max': dEmax, 'energy_error_eh_mean': sum(dE) / len(dE),
                  'energy_error_eh_per_molecule': dE},
        'algorithmic_tflops': flops / t_dev / 1e12,
        'grid_points_per_s': sum(sum(r * a for r, a in zip(m['nrad'], m['nang']))
                                 for m in all_mols) / t_dev,
        'setup_s': t_setup,
        'clocks': clk8 if ok else clk64,
        'cpu_baseline': None,
    }
    if rank == 0:
        print(json.dumps(line))


# ------------------------------------------------------- C5: gradients
def run_gradients(args, world, rank):
    """H2O with both protons quantum (5s5p nuclear basis), 75 x 194 Becke grid
    per centre.  For 32 seeded geometries (each coordinate perturbed uniformly
    within +-0.05 A): for the electrons and for the protons, the grid
    quadrature energy in the potential of the classical O nucleus, dE/dD (the
    quadrature matrix) and dE/dR (hand-written gradient kernel).  One step =
    the 32 geometries x 2 species; the first geometry is checked against
    central differences (h = 1e-4 bohr)."""
    import torch
    from napmo_b200.gradients import GridChargeEnergy
    from napmo_b200.system import BOHR_TO_ANGSTROM
    sym = ['O', 'H', 'H']
    R0 = np.array([(0.0, 0.0, 0.0), (0.0, 0.757, 0.587), (0.0, -0.757, 0.587)])
    rng = np.random.default_rng(SEED)
    geoms = [(R0 + rng.uniform(-0.05, 0.05, size=R0.shape)) / BOHR_TO_ANGSTROM
             for _ in range(32)]
    models = [GridChargeEnergy(sym, species=sp, quantum=(1, 2), nrad=75, nang=194)
              for sp in ('e-', 'H_1')]
    dens = {}
    for m in models:
        V, _ = m.quadrature_matrix(geoms[0])
        n = V.shape[0]
        C = np.random.default_rng(SEED + n).normal(size=(n, 5 if m.species == 'e-' else 2))
        dens[m.species] = 2.0 * C @ C.T / n if m.species == 'e-' else C @ C.T / n

    def one_pass():
        out = []
        for R in geoms:
            for m in models:
                V, st = m.quadrature_matrix(R)
                E, g = m.gradient(st, dens[m.species])
                out.append((E, g))
        return out

    for _ in range(max(1, args.warmup)):
        one_pass()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res = one_pass()
    torch.cuda.synchronize()
    t_step = (time.perf_counter() - t0) / args.steps
    # gradient kernel alone (device events), first geometry
    kern = {}
    for m in models:
        V, st = m.quadrature_matrix(geoms[0])
        m.gradient(st, dens[m.species])
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(5):
            m.gradient(st, dens[m.species])
        ev1.record()
        ev1.synchronize()
        kern[m.species] = {'ms': ev0.elapsed_time(ev1) / 5, 'npoint': st['grid'].size,
                           'nbasis': V.shape[0]}
    # central differences, first geometry
    fd = {}
    h = 1e-4
    for m in models:
        D = dens[m.species]
        V, st = m.quadrature_matrix(geoms[0])
        _, g = m.gradient(st, D)
        gf = np.zeros_like(g)
        for a in range(3):
            for k in range(3):
                Rp, Rm = geoms[0].copy(), geoms[0].copy()
                Rp[a, k] += h
                Rm[a, k] -= h
                Ep = float((D * m.quadrature_matrix(Rp)[0].cpu().numpy()).sum())
                Em = float((D * m.quadrature_matrix(Rm)[0].cpu().numpy()).sum())
                gf[a, k] = (Ep - Em) / (2 * h)
        fd[m.species] = {'max_abs_error_eh_per_bohr': float(np.abs(g - gf).max()),
                         'max_abs_gradient': float(np.abs(gf).max()),
                         'net_force': float(np.abs(g.sum(axis=0)).max())}
    # int8 quadrature matrices (dE/dD) against FP64 over the geometries; the
    # gradient kernel runs in FP64 in both modes
    mixed = {}
    for m in models:
        m8 = GridChargeEnergy(sym, species=m.species, quantum=(1, 2), nrad=75, nang=194,
                              precision='int8x4')
        D = dens[m.species]
        dV, dE, dg = 0.0, 0.0, 0.0
        for R in geoms:
            V, st = m.quadrature_matrix(R)
            V8, st8 = m8.quadrature_matrix(R)
            V, V8 = V.cpu().numpy(), V8.cpu().numpy()
            dV = max(dV, float(np.abs(V8 - V).max() / np.abs(V).max()))
            dE = max(dE, abs(float((D * (V8 - V)).sum())))
            dg = max(dg, float(np.abs(m8.gradient(st8, D)[1] - m.gradient(st, D)[1]).max()))
        mixed[m.species] = {'max_rel_dEdD_error': dV, 'max_energy_error_eh': dE,
                            'max_gradient_error_eh_per_bohr': dg}
    nunit = len(geoms) * len(models)
    line = {
        'metric': 'grid energy gradients/s (H2O, both protons quantum, 75x194; C5)',
        'value': nunit / t_step, 'unit': 'gradients/s', 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': t_step * 1e3, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': 'C5: 32 seeded geometries (+-0.05 A) x {electrons, protons}; '
                               'grid, basis, quadrature and gradient per geometry',
                   'parallelism': 'single GPU'},
        'gradient_kernel': kern,
        'finite_differences': fd,
        'mixed_int8x4': mixed,
        'e2e': {'value': nunit / t_step, 'unit': 'gradients/s',
                'h2d_bytes_per_step': sum(8 * dens[m.species].size for m in models) * len(geoms),
                'd2h_bytes_per_step': 8 * 10 * nunit},
        'cpu_baseline': None,
    }
    if rank == 0:
        print(json.dumps(line))


# ---------------------------------------------------------- C1: grid SCF
def run_scf_c1(args, world, rank):
    """H2O / cc-pVDZ (O at 0, H at (0, +-0.757, 0.587) A), 50 x 110 Becke
    grid, closed-shell SCF with J and exchange on the grid (orbital-pair
    Poisson solves), DIIS with 6 vectors, converged to 1e-8 Eh; one step = one
    SCF from the core guess.  FP64 and int8x4 contractions."""
    import torch
    from napmo_b200.scf import GridRHF
    from napmo_b200.system import build_system
    atoms = [('O', (0.0, 0.0, 0.0)), ('H', (0.0, 0.757, 0.587)), ('H', (0.0, -0.757, 0.587))]
    out, clocks = {}, {}
    for prec in ('fp64', 'int8x4'):
        times, res = [], None
        sampler = ClockSampler(torch.cuda.current_device())
        for k in range(args.warmup + args.steps):
            scf = GridRHF(build_system(atoms, 'CC-PVDZ'), 50, 110, exchange='hf',
                          precision=prec)
            if k == args.warmup:
                sampler.start()
            res = scf.run(tol=1e-8)
            if k >= args.warmup:
                times.append(res['seconds'])
        clocks[prec] = sampler.stop()
        out[prec] = {'seconds': statistics.median(times), 'energy': res['energy'],
                     'iterations': res['iterations'], 'converged': res['converged'],
                     'fock_builds': res['fock_builds'], 'poisson_solves': res['poisson_solves']}
    dE = abs(out['int8x4']['energy'] - out['fp64']['energy'])
    head = 'int8x4' if dE <= 1e-6 and out['int8x4']['converged'] else 'fp64'
    t = out[head]['seconds']
    line = {'metric': 'grid RHF SCF time, H2O / cc-pVDZ 50x110 (C1)', 'value': t,
            'unit': 's per SCF', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': t * 1e3, 'higher_is_better': False, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'int8x4' if head == 'int8x4' else 'f64',
            'data': 'synthetic',
            'config': {'workload': 'C1: H2O cc-pVDZ (25 Cartesian functions), 50x110 per atom '
                                   '(16,500 points), lmax 8, grid J and exchange, DIIS(6), 1e-8 Eh',
                       'parallelism': 'single GPU'},
            'scf': out, 'energy_difference_eh': dE, 'clocks': clocks[head],
            'e2e': {'value': t, 'unit': 's per SCF', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 8},
            'cpu_baseline': None}
    if rank == 0:
        print(json.dumps(line))


# -------------------------------------------------------- C2: APMO SCF
def run_scf_c2(args, world, rank):
    """HCN (H at 0, C at 1.066 A, N at 2.222 A along z), electrons in
    cc-pVDZ, the H nucleus as a quantum species (5s5p even-tempered, 4-64
    bohr^-2), 100 x 302 Becke grid per atom (90,600 points) shared by both
    species; electron-nucleus coupling by grid quadrature of the device
    Poisson potentials, electron exchange from orbital-pair Poisson solves,
    one DIIS (6) over both species, converged to 1e-8 Eh."""
    import torch
    from napmo_b200.scf import GridAPMO
    from napmo_b200.system import build_system
    atoms = [('H', (0.0, 0.0, 0.0)), ('C', (0.0, 0.0, 1.066)), ('N', (0.0, 0.0, 2.222))]
    out, clocks = {}, {}
    for prec in ('fp64', 'int8x4'):
        times, res = [], None
        sampler = ClockSampler(torch.cuda.current_device())
        for k in range(args.warmup + args.steps):
            ms = build_system(atoms, 'CC-PVDZ', quantum=(0,))
            drv = GridAPMO(ms, 'H_1', 100, 302, precision=prec)
            if k == args.warmup:
                sampler.start()
            res = drv.run(tol=1e-8)
            if k >= args.warmup:
                times.append(res['seconds'])
        clocks[prec] = sampler.stop()
        out[prec] = {'seconds': statistics.median(times), 'energy': res['energy'],
                     'iterations': res['iterations'], 'converged': res['converged'],
                     'poisson_solves': res['poisson_solves']}
    dE = abs(out['int8x4']['energy'] - out['fp64']['energy'])
    head = 'int8x4' if dE <= 1e-6 and out['int8x4']['converged'] else 'fp64'
    t = out[head]['seconds']
    line = {'metric': 'grid APMO-RHF SCF time, HCN with quantum H, 100x302 (C2)', 'value': t,
            'unit': 's per SCF', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': t * 1e3, 'higher_is_better': False, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'int8x4' if head == 'int8x4' else 'f64',
            'data': 'synthetic',
            'config': {'workload': 'C2: HCN, e- cc-pVDZ (35) + H nucleus 5s5p (20), 100x302 per '
                                   'atom (90,600 points), lmax 14, DIIS(6), 1e-8 Eh',
                       'parallelism': 'single GPU'},
            'scf': out, 'energy_difference_eh': dE, 'clocks': clocks[head],
            'e2e': {'value': t, 'unit': 's per SCF', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 8},
            'cpu_baseline': None}
    if rank == 0:
        print(json.dumps(line))


# ------------------------------------------- C6: Becke-Dickson numerical HF
C6_ATOMS = [('He', (0.0, 0.0, 0.0))]
# iterations of the C6 SCF (the same on the host: the reference arm times
# nAPMO's algorithm for the same number of optimiser steps)
C6_REF_ITERATIONS = 12
C6_WORKLOAD = ('C6: He, numerical orbitals on a 300x110 Becke grid (33,000 points, lmax 8) '
               'started from STO-3G; Becke-Dickson optimiser + grid Fock step per iteration '
               'until |dE| < 1e-8 Eh (napmo/wavefunction/test/test_psi_numeric_becke_He.py)')


def c6_cpu_baseline(iterations):
    """nAPMO's numerical-orbital iteration restated on the host (oracle):
    one kinetic operator, one Becke-Dickson correction and one Poisson solve
    timed on the He 300x110 grid, scaled to one iteration's counts (3 kinetic
    images, 1 correction, 5 Poisson solves) and to the SCF's iterations."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import numeric as ON
    import oracle as O
    el = json.load(open(os.path.join(ROOT, 'napmo_b200', 'data', 'elements.json')))
    g = O.Grid([np.zeros(3)], [el['He']['atomic_radii']], 300, 110)
    r2 = (g.points ** 2).sum(1)
    psi = np.exp(-1.3 * r2)
    vnuc = 2.0 / np.sqrt(r2)
    t0 = time.perf_counter()
    T = ON.compute_kinetic(g, psi, 8)
    t1 = time.perf_counter()
    ON.compute_dpsi(g, 8, psi, 0.01, -0.9, 0.05 * T, -psi * vnuc, 1.0)
    t2 = time.perf_counter()
    O.compute_coulomb(g, 2.0 * psi * psi, 8)
    t3 = time.perf_counter()
    per_it = 3 * (t1 - t0) + (t2 - t1) + 5 * (t3 - t2)
    return {'value': per_it * iterations, 'unit': 's per SCF', 'cores': O.threads(),
            'kind': 'port',
            'sample': 'one kinetic image (%.3f s), one Becke-Dickson correction (%.3f s), one '
                      'Poisson solve (%.3f s) on He 300x110, scaled to 3/1/5 per iteration x %d '
                      'iterations' % (t1 - t0, t2 - t1, t3 - t2, iterations),
            'seconds_per_iteration': per_it}


def run_becke_c6(args, world, rank):
    """He numerical HF through PSIN + PSIO_BECKE on the device; one step =
    one Becke-Dickson SCF from the STO-3G orbitals (the basis-set SCF that
    provides them is not timed)."""
    import torch
    from napmo_b200.numeric import GridOperators, from_grid_rhf, optimize
    from napmo_b200.scf import GridRHF
    from napmo_b200.system import build_system
    rhf = GridRHF(build_system(C6_ATOMS, 'STO-3G'), 300, 110, exchange='hf')
    gto = rhf.run(tol=1e-10)
    times, res = [], None
    sampler = ClockSampler(torch.cuda.current_device())
    for k in range(args.warmup + args.steps):
        psin = from_grid_rhf(rhf)
        if k == args.warmup:
            sampler.start()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = optimize(psin, tol=1e-8)
        torch.cuda.synchronize()
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    t = statistics.median(times)
    its = res['iterations']
    # device time of the operators of one iteration (CUDA events)
    ops = GridOperators(rhf.grid, 8)
    psi2 = torch.cat([psin.psi, psin.optimizer.delta_psi])
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    ops.kinetic(psi2, 1.0)
    ev[1].record()
    ops.dpsi(psin.psi, psin.Tgrid, psin.Vgrid, [0.01], [-0.9], 1.0)
    ev[2].record()
    ops.coulomb(psin.Dgrid.sum(0))
    ev[3].record()
    torch.cuda.synchronize()
    parts = {'kinetic_2_functions_ms': ev[0].elapsed_time(ev[1]),
             'becke_dickson_1_orbital_ms': ev[1].elapsed_time(ev[2]),
             'poisson_ms': ev[2].elapsed_time(ev[3])}
    cb = c6_cpu_baseline(its) if not args.no_cpu_baseline and rank == 0 else None
    line = {'metric': 'Becke-Dickson numerical HF time, He 300x110 (C6)', 'value': t,
            'unit': 's per SCF', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': t * 1e3, 'higher_is_better': False, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': C6_WORKLOAD, 'parallelism': 'single GPU',
                       'l2': 'inputs (33,000-point orbital images) stay resident; the SCF is '
                             'launch- and host-step bound, not HBM bound'},
            'energy': res['energy'], 'iterations': its, 'converged': res['converged'],
            'gto_energy': gto['energy'], 'ms_per_iteration': t * 1e3 / its,
            'device_parts': parts, 'clocks': clocks,
            'e2e': {'value': t, 'unit': 's per SCF', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 8 * its},
            'cpu_baseline': cb}
    if rank == 0:
        print(json.dumps(line))


# ----------------------------------------- C7: one-electron integrals on the GPU
C7_WORKLOAD = ('C7: S, T and V = -sum Z <1/r_C> of C20H42/cc-pVDZ (510 Cartesian functions, '
               '130,305 pairs, 62 point charges), nAPMO\'s libint one-body calls')


def c7_cpu_baseline(ms):
    """The host restatements: S and T by the product's host Obara-Saika code
    (C++, one thread, all pairs); V by the oracle (McMurchie-Davidson in
    Python) on a sample of 400 function pairs, scaled to all pairs."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import ints as OI
    from napmo_b200 import cext
    b = ms['e-']['basis']
    n = b['nbasis']
    S, T = np.zeros((n, n)), np.zeros((n, n))
    t0 = time.perf_counter()
    cext.checked(cext.lib.napmo_basis_one_body(b._this, S, T))
    t_st = time.perf_counter() - t0
    rng = np.random.default_rng(SEED)
    pairs = rng.integers(0, n, size=(400, 2))
    charges = [(pc['atomic_number'], np.asarray(pc['origin'])) for pc in ms.point_charges]
    cont = b['cont']
    t0 = time.perf_counter()
    for i, j in pairs:
        ci, cj = cont[i], cont[j]
        li, lj, oi, oj = [int(x) for x in ci.l], [int(x) for x in cj.l], ci.origin, cj.origin
        for pa in ci._primitives:
            for pb in cj._primitives:
                OI.primitive(li, oi, pa.exponent, lj, oj, pb.exponent, charges)
    t_v = (time.perf_counter() - t0) * (n * (n + 1) / 2) / len(pairs)
    return {'value': t_st + t_v, 'unit': 's per S,T,V', 'cores': 1, 'kind': 'port',
            'sample': 'S, T: all pairs by the host C++ code (%.3f s); V: 400 seeded pairs by the '
                      'oracle, scaled to 130,305 pairs (%.1f s)' % (t_st, t_v)}


def run_ints_c7(args, world, rank):
    import torch
    from napmo_b200 import cext
    from napmo_b200.system import alkane_geometry, build_system
    ms = build_system(alkane_geometry(20), 'CC-PVDZ')
    b = ms['e-']['basis']
    n = b['nbasis']
    q = np.ascontiguousarray(np.array([[*pc['origin'], pc['atomic_number']]
                                       for pc in ms.point_charges], dtype=np.float64))
    out = [torch.empty((n, n), dtype=torch.float64, device='cuda') for _ in range(3)]
    stream = torch.cuda.current_stream()

    def one():
        cext.checked(cext.lib.napmo_gpu_one_body(b._this, q.shape[0], q.ctypes.data,
                                                 *[o.data_ptr() for o in out],
                                                 stream.cuda_stream))
    for _ in range(args.warmup):
        one()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(args.steps):
        one()
    ev[1].record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    t = ev[0].elapsed_time(ev[1]) / 1e3 / args.steps
    cb = c7_cpu_baseline(ms) if not args.no_cpu_baseline and rank == 0 else None
    line = {'metric': 'one-electron integrals S, T, V of C20H42/cc-pVDZ (C7)', 'value': t,
            'unit': 's per S,T,V', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': t * 1e3, 'higher_is_better': False, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': C7_WORKLOAD, 'parallelism': 'single GPU',
                       'l2': 'inputs are the basis description (a few KB); outputs 6 MB'},
            'clocks': clocks, 'gpu_launches': args.steps,
            'e2e': {'value': t, 'unit': 's per S,T,V', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0},
            'cpu_baseline': cb}
    if rank == 0:
        print(json.dumps(line))


# --------------------------------------------------------------------- main
def main():
    args = parse()
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', str(args.gpus)))
    local = int(os.environ.get('LOCAL_RANK', '0'))

    if args.impl == 'reference':
        if rank != 0:
            return
        if args.workload in ('c1', 'c2'):
            print(json.dumps(reference_scf(args, args.workload)))
            return
        why = {'c3': 'nAPMO has no batched multi-molecule build; its per-build CPU cost is the '
                     'c4 reference arm',
               'c5': 'nAPMO computes no nuclear-coordinate gradients'}
        if args.workload in why:
            print(json.dumps({'impl': 'reference', 'workload': args.workload,
                              'unavailable': why[args.workload]}))
            return
        if args.workload == 'c7':
            from napmo_b200.system import alkane_geometry, build_system
            ms = build_system(alkane_geometry(20), 'CC-PVDZ')
            vals, cb = [], None
            for _ in range(args.warmup + args.steps):
                cb = c7_cpu_baseline(ms)
                vals.append(cb['value'])
            v = statistics.median(vals[args.warmup:])
            cb['value'] = v
            print(json.dumps({
                'impl': 'reference', 'metric': 'one-electron integrals S, T, V of C20H42/cc-pVDZ (C7)',
                'value': v, 'unit': 's per S,T,V', 'n_gpus': 1, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': v * 1e3, 'higher_is_better': False,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
                'config': {'workload': C7_WORKLOAD, 'parallelism': 'host, one thread'},
                'cpu_baseline': cb,
                'e2e': {'value': v, 'unit': 's per S,T,V', 'h2d_bytes_per_step': 0,
                        'd2h_bytes_per_step': 0}}))
            return
        if args.workload == 'c6':
            vals, cb = [], None
            for _ in range(args.warmup + args.steps):
                cb = c6_cpu_baseline(C6_REF_ITERATIONS)
                vals.append(cb['value'])
            v = statistics.median(vals[args.warmup:])
            cb['value'] = v
            print(json.dumps({
                'impl': 'reference', 'metric': 'Becke-Dickson numerical HF time, He 300x110 (C6)',
                'value': v, 'unit': 's per SCF', 'n_gpus': 1, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': v * 1e3, 'higher_is_better': False,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
                'config': {'workload': C6_WORKLOAD, 'parallelism': 'host cores'},
                'cpu_baseline': cb,
                'e2e': {'value': v, 'unit': 's per SCF', 'h2d_bytes_per_step': 0,
                        'd2h_bytes_per_step': 0}}))
            return
        # the host arm loads no part of this package's library: the oracle
        # builds the grid, the sample and the density
        hw = HostWorkload(args)
        steps = []
        for _ in range(args.warmup + args.steps):
            cb = cpu_baseline(args, hw)
            steps.append(cb)
        timed = steps[args.warmup:]
        v = statistics.median([c['value'] for c in timed])
        sample_s = statistics.median([c['sample_seconds'] for c in timed])
        cb['value'] = v
        line = {'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': UNIT, 'n_gpus': world,
                'steps': args.steps, 'warmup': args.warmup,
                # what each step actually ran; value is that sample scaled to a build
                'ms_per_step': sample_s * 1e3,
                'sample_scale_to_build': (1.0 / v) / sample_s,
                'extrapolated_ms_per_build': 1e3 / v,
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
                'dtype': 'f64', 'data': 'synthetic',
                'config': c4_config(world, hw.n, hw.N, hw.lmax),
                'cpu_baseline': cb,
                'e2e': {'value': v, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                        'd2h_bytes_per_step': 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    import napmo_b200 as nb
    from napmo_b200 import cext

    if args.workload in ('c3', 'c5', 'c1', 'c2', 'c6', 'c7'):
        if args.workload == 'c3':
            run_batch(args, world, rank, dist)
        else:
            {'c5': run_gradients, 'c1': run_scf_c1, 'c2': run_scf_c2,
             'c6': run_becke_c6, 'c7': run_ints_c7}[args.workload](
                args, world, rank)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    atoms, ms, grid, basis, lmax, D = build_workload(args)
    n = basis['nbasis']
    N = grid.size
    fbld = nb.FockBuilder(grid, basis, lmax)
    Dd = torch.as_tensor(D, device='cuda')
    stream = torch.cuda.current_stream()
    F = torch.empty((n, n), dtype=torch.float64, device='cuda')

    def timed_builds(precision, screen=0.0, poisson_tol=None):
        fbld.set_precision(precision)
        if precision == 'fp64':
            fbld.set_fp64_screening(screen)
        if poisson_tol is not None:
            fbld.set_poisson_tolerance(poisson_tol)
        for _ in range(args.warmup):
            fbld.build(Dd, out=F)
        torch.cuda.synchronize()
        sampler = ClockSampler(torch.cuda.current_device())
        sampler.start()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            fbld.build(Dd, out=F)
        ev1.record(stream)
        ev1.synchronize()
        t = ev0.elapsed_time(ev1) / 1e3
        clk = sampler.stop()
        if dist:
            tt = torch.tensor([t], device='cuda')
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = tt.item()
        E = 0.5 * float((F * Dd).sum())
        return t, clk, E

    t_f64, clocks_f64, E_f64 = timed_builds('fp64')
    F64 = F.clone()
    # the FP64 arm with the int8 mode's two precision-independent savings:
    # point screening (1e-24) and the Poisson truncation (1e-9 a.u.)
    t_f64s, _, E_f64s = timed_builds('fp64', screen=1e-24, poisson_tol=1e-9)
    fbld.set_fp64_screening(0.0)
    t_tc, clocks_tc, E_tc = timed_builds('int8x4')
    tc_err = fbld.tc_status()
    dE = abs(E_tc - E_f64)
    mixed_ok = (tc_err == 0) and dE <= 1e-6
    headline = 'int8x4' if (mixed_ok and args.precision != 'fp64') else 'fp64'
    fbld.set_precision(headline)
    t_dev = t_tc if headline == 'int8x4' else t_f64
    clocks = clocks_tc if headline == 'int8x4' else clocks_f64
    # kernels per build: density (FP64: 1; int8: slice D + density), Poisson
    # (project, radial, pair evaluation, pair reduce), weights, quadrature
    # (FP64: GEMM + reduce; int8: slice wv phi + GEMM + reduce)
    launches_per_build = 9 if headline == 'int8x4' else 8
    mixed = {'builds_per_s': world * args.steps / t_tc, 'ms_per_build': t_tc / args.steps * 1e3,
             'energy_error_eh': dE, 'max_abs_dF': float((F - F64).abs().max()),
             'speedup_vs_fp64': t_f64 / t_tc, 'tc_status': tc_err,
             'int8_image_bytes': int(cext.lib.napmo_fock_plan_int8_bytes(fbld._plan)),
             'scheme': 'int8 slices (4 balanced base-256 digits per value, group exponents), '
                       'tcgen05 kind::i8 with exact int32 TMEM accumulation; 13 digit '
                       'products per contraction; Poisson FP64, its evaluation skipping '
                       'l-blocks bounded below 1e-9 a.u. per (atom, radial interval)'}

    # ---- per-kernel timings (same stream) for the roofline
    def time_it(fn, reps=3):
        fn()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record(stream)
        for _ in range(reps):
            fn()
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e) / 1e3 / reps

    rho = fbld.density(Dd)
    v = fbld.coulomb_potential(rho)
    flops = 2.0 * n * n * N
    kernels = {}
    for prec in ('fp64', 'int8x4'):
        fbld.set_precision(prec)
        td = time_it(lambda: fbld.density(Dd))
        tq = time_it(lambda: fbld.quadrature(1.0, v))
        kernels['density_' + prec] = {'ms': td * 1e3, 'tflops': flops / td / 1e12}
        kernels['quadrature_' + prec] = {'ms': tq * 1e3, 'tflops': flops / tq / 1e12}
        # projection + radial solves + evaluation; int8x4 evaluates with the
        # mode's truncation tolerance (l-blocks bounded below 1e-9 skipped)
        tp = time_it(lambda: fbld.coulomb_potential(rho))
        kernels['poisson_' + prec] = {'ms': tp * 1e3}
    fbld.set_precision(headline)
    t_density = kernels['density_' + headline]['ms'] / 1e3
    t_quad = kernels['quadrature_' + headline]['ms'] / 1e3
    t_poisson_mode = kernels['poisson_' + headline]['ms'] / 1e3

    # ---- end-to-end through the C-ABI with host buffers
    Dh = torch.empty((n, n), dtype=torch.float64).pin_memory()
    Dh.copy_(torch.as_tensor(D))
    Fh = torch.empty((n, n), dtype=torch.float64).pin_memory()
    Dn, Fn = Dh.numpy(), Fh.numpy()
    for _ in range(2):
        cext.checked(cext.lib.napmo_fock_plan_build_host(fbld._plan, Dn, 1.0, None, Fn,
                                                         stream.cuda_stream))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cext.checked(cext.lib.napmo_fock_plan_build_host(fbld._plan, Dn, 1.0, None, Fn,
                                                         stream.cuda_stream))
    t_e2e = time.perf_counter() - t0
    if dist:
        t = torch.tensor([t_e2e], device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = t.item()

    # ---- SCF of C20H42 (Slater exchange on the grid; J by the same Fock builds)
    scf = None
    if not args.no_scf:
        from napmo_b200.scf import GridRHF
        scf = {}
        for prec in ('fp64', 'int8x4'):
            run = GridRHF(ms, args.nrad, args.nang, lmax=lmax, exchange='lda-x', precision=prec)
            res = run.run(tol=1e-7)
            scf[prec] = {'seconds': res['seconds'], 'energy': res['energy'],
                         'iterations': res['iterations'], 'converged': res['converged'],
                         'fock_builds': res['fock_builds']}
            del run
        scf['energy_difference_eh'] = abs(scf['int8x4']['energy'] - scf['fp64']['energy'])
        scf['model'] = 'closed-shell SCF, J and Slater exchange on the grid, DIIS(6), 1e-7 Eh'

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        fp64 = fp64_gemm_peak(torch)
        stages = {'density': t_density, 'quadrature': t_quad, 'poisson': t_poisson_mode}
        dom = max(stages, key=stages.get)
        td = stages[dom]
        if dom == 'poisson':
            # the roofline is the kernel's: the untruncated evaluation, whose
            # work is the full (l, m) count below
            td = kernels['poisson_fp64']['ms'] / 1e3
        issued = None
        if dom == 'poisson':
            # potential evaluation dominates: FP64 ALU bound.  Algorithmic count:
            # 20 flops per (atom, point, lm) as nAPMO evaluates it; the kernel
            # executes about 10.5 L(L+1) + 11 (L+1) + 3 L + 20 flops per
            # (atom, point): per (l, m > 0) the rescaled recursion (3), the two
            # products with cos/sin (2) and two 4-coefficient terms (16).
            natom = len(atoms)
            lsize = (lmax + 1) ** 2
            flops_alg = 20.0 * natom * lsize * N
            flops_exec = (10.5 * lmax * (lmax + 1) + 11.0 * (lmax + 1) + 3.0 * lmax + 20.0) * natom * N
            achieved = flops_alg / td / 1e12
            peak = fp64
            bound = 'fp64'
            peak_source = ('FP64: cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json lists '
                           'HBM/bf16 only); stage = projection + radial + evaluation + reduce (FP64 '
                           'mode, untruncated), the evaluation kernel is 94 % of it (launch list). '
                           'frac exceeds 1 because the algorithmic count is 20 flops per (pair, lm) '
                           'while the kernel executes about 10.5: see issued')
            issued = {'executed_fp64_tflops': flops_exec / td / 1e12,
                      'frac_executed': flops_exec / td / 1e12 / fp64}
            kernel_name = 'poisson(eval_pairs dominant)'
            # DRAM bytes of the evaluation per launch: 29.9 B per (atom, point)
            # pair (ncu at C8H18: 0.61 GB for 20.4 M pairs; pair lists, stored
            # u and 1/d and partial potentials grow with the pairs)
            traffic = EVAL_DRAM_BYTES_PER_PAIR * natom * N
        else:
            traffic = None
            flops_alg = flops
            achieved = flops / td / 1e12
            bound = 'tensor'
            kernel_name = dom + '_' + headline
            nprod = 13
            if headline == 'int8x4':
                peak = 2.0 * float(peaks.get('bf16_tflops', 1590.0))
                peak_source = ('int8 dense = 2 x bf16 dense burst (%s); the scheme issues %d int8 '
                               'MMAs per algorithmic FLOP, so frac <= 1/%d at full tensor '
                               'throughput' % (peak_kind, nprod, nprod))
                issued = {'int8_tops': nprod * achieved,
                          'frac_of_int8_peak': nprod * achieved / peak}
            else:
                peak = fp64
                peak_source = ('cuBLAS DGEMM 8192^3 measured in this run (FP64; the peaks file '
                               'lists HBM/bf16 only)')
        value = world * args.steps / t_dev
        cb = None
        if not args.no_cpu_baseline and world == 1:
            cb = cpu_baseline(args, HostWorkload(args))
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': t_dev / args.steps * 1e3,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'int8x4' if headline == 'int8x4' else 'f64', 'data': 'synthetic',
            'config': c4_config(world, n, N, lmax),
            'e2e': {'value': world * args.steps / t_e2e, 'unit': UNIT,
                    'h2d_bytes_per_step': n * n * 8, 'd2h_bytes_per_step': n * n * 8},
            'gpu_launches': launches_per_build * args.steps,
            'roofline': {'kernel': kernel_name, 'bound': bound, 'achieved': achieved,
                         'peak': peak, 'unit': 'TFLOP/s', 'frac': achieved / peak,
                         'traffic': traffic, 'traffic_source': TRAFFIC_SOURCE if traffic else None,
                         'peak_source': peak_source,
                         'algorithmic_flops_per_launch': flops_alg, 'issued': issued},
            'stages_ms': {k: v * 1e3 for k, v in stages.items()},
            'grid_points_per_s': world * args.steps / t_dev * N,
            'fp64': {'builds_per_s': world * args.steps / t_f64,
                     'ms_per_build': t_f64 / args.steps * 1e3, 'fp64_gemm_tflops': fp64},
            'fp64_screened_truncated': {
                'builds_per_s': world * args.steps / t_f64s,
                'ms_per_build': t_f64s / args.steps * 1e3,
                'energy_difference_eh': abs(E_f64s - E_f64),
                'mixed_speedup_vs_this_arm': t_f64s / t_tc,
                'note': 'FP64 contractions with the int8 mode\'s point screening (1e-24) and '
                        'Poisson truncation (1e-9 a.u.): the speed-up over this arm is the '
                        'tensor cores\' share'},
            'mixed': mixed,
            'kernels': kernels,
            'scf': scf,
            'clocks': clocks,
            'cpu_baseline': cb,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
