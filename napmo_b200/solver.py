"""Solvers with the interface of nAPMO's napmo.solver (HF: hf_solver.py:15-146,
DFT: dft_solver.py:15-137): ``HF(system, options).compute()`` returns the
total energy, with every grid quadrature, Poisson solve and contraction on
the device.

nAPMO's analytic ('kind': 'analytic') solvers take S, T, V and the
two-electron integrals from libint; here the same SCF runs on the grid (S, T
analytic, V_ne, J, exchange and the coupling of species by grid quadrature of
device Poisson potentials) through the drivers of napmo_b200.scf:

  electrons only, closed shell       GridRHF    (RHF)
  electrons only, open shell / 'uhf' GridUHF    (e-alpha and e-beta)
  one quantum-nucleus species        GridAPMO   (APMO-RHF)
    ... with open-shell electrons    GridMultiSCF (APMO-UHF)

'kind': 'numeric' with electrons only runs nAPMO's numerical-orbital
Becke-Dickson SCF (PSIN + PSIO_BECKE, psi_numeric.py / psi_optimization.py)
from the grid RHF orbitals.

Options (nAPMO's names): 'method' ('hf', 'rhf', 'uhf', 'dft'), 'kind',
'grid' ([nrad, nang] or {'e-': {'nrad': .., 'nang': ..}}), 'maxiter',
'eps_e' (energy change at convergence), and for DFT 'functional'
({'e-': 'lda', 'e-:H_1': 'epc17-2'}).  Added here: 'precision' ('fp64' or
'int8x4' for rho and the quadratures) and 'diis' (vectors).
"""
from . import scf as _scf

_DEFAULTS = {'maxiter': 100, 'eps_e': 1e-7, 'kind': 'analytic', 'grid': [100, 110],
             'precision': 'fp64', 'diis': 6}


def _grid(options):
    g = options.get('grid', [100, 110])
    if isinstance(g, dict):
        e = g.get('e-', {})
        return int(e.get('nrad', 100)), int(e.get('nang', 110))
    return int(g[0]), int(g[1])


class _Solver(object):

    def __init__(self, system, options=None, pprint=True):
        self.system = system
        self.options = dict(_DEFAULTS, **self._defaults())
        if options:
            self.options.update(options)
        self.pprint = pprint
        self._energy = 0.0
        self.result = None

    def _defaults(self):
        return {}

    def get(self, key, default=None):
        return self.options.get(key, default)

    def _quantum(self):
        q = [k for k in self.system if k != 'e-']
        if len(q) > 1:
            raise NotImplementedError('one quantum-nucleus species is supported')
        return q[0] if q else None

    def _open_shell(self):
        """nAPMO's set_charges runs for every input: an odd electron count or a
        multiplicity above 1 splits the electrons into alpha and beta."""
        if self.get('method') == 'uhf' or getattr(self.system, 'open_shell', False):
            return True
        nel = int(round(self.system['e-']['size'])) - self._charge()
        m = self._multiplicity() or (nel % 2) + 1
        return m > 1

    def _charge(self):
        # nAPMO's e- charge counts added electrons; the drivers take the
        # molecular charge
        return -int(getattr(self.system, 'charges', {}).get('e-', {}).get('charge', 0))

    def _multiplicity(self):
        return getattr(self.system, 'charges', {}).get('e-', {}).get('multiplicity') or None

    def _run(self, driver):
        res = driver.run(maxiter=int(self.get('maxiter')), tol=float(self.get('eps_e')),
                         verbose=self.pprint)
        self.driver, self.result = driver, res
        self._energy = res['energy']
        if self.pprint:
            print('%-11s %16.10f  (%d iterations)' % ('TOTAL', self._energy, res['iterations']))
        return self._energy

    @property
    def energy(self):
        return self._energy


class HF(_Solver):
    """Hartree-Fock (or APMO-HF with one quantum-nucleus species) on the grid."""

    def _defaults(self):
        return {'method': 'hf'}

    def compute(self, pprint=None):
        if pprint is not None:
            self.pprint = pprint
        nrad, nang = _grid(self.options)
        nuc = self._quantum()
        kw = dict(precision=self.get('precision'), diis=int(self.get('diis')))
        if self.get('kind') == 'numeric':
            if nuc is not None or self._open_shell():
                raise NotImplementedError('numerical orbitals: closed-shell electrons only')
            return self._numeric(nrad, nang, kw)
        if nuc is None:
            if self._open_shell():
                drv = _scf.GridUHF(self.system, nrad, nang, charge=self._charge(),
                                   multiplicity=self._multiplicity(), **kw)
            else:
                drv = _scf.GridRHF(self.system, nrad, nang, exchange='hf', **kw)
        elif self._open_shell():
            drv = _scf.GridMultiSCF(self.system, nuc, nrad, nang, charge=self._charge(),
                                    multiplicity=self._multiplicity(), **kw)
        else:
            drv = _scf.GridAPMO(self.system, nuc, nrad, nang, **kw)
        return self._run(drv)

    def _numeric(self, nrad, nang, kw):
        """Grid RHF orbitals, then nAPMO's Becke-Dickson optimisation of the
        numerical orbitals (PSIN / PSIO_BECKE) on the same grid."""
        from .numeric import from_grid_rhf, optimize
        rhf = _scf.GridRHF(self.system, nrad, nang, exchange='hf', **kw)
        self._run(rhf)
        self.psin = from_grid_rhf(rhf)
        res = optimize(self.psin, maxiter=int(self.get('maxiter')), tol=float(self.get('eps_e')),
                       verbose=self.pprint)
        self.result = res
        self._energy = res['energy']
        return self._energy


class DFT(_Solver):
    """Kohn-Sham DFT on the grid: the electrons' functional ('lda': Slater
    exchange + VWN5 correlation) and, with a quantum-nucleus species, the
    electron-nucleus correlation functional of the pair key 'e-:<nucleus>'
    (or '<nucleus>:e-'), e.g. 'epc17-2'."""

    def _defaults(self):
        return {'method': 'dft', 'functional': {'e-': 'lda'}}

    def compute(self, pprint=None):
        if pprint is not None:
            self.pprint = pprint
        nrad, nang = _grid(self.options)
        nuc = self._quantum()
        func = dict(self.get('functional') or {})
        xc = func.get('e-', 'lda')
        if xc != 'lda':
            raise NotImplementedError(str(xc) + ' Functional NOT available!')
        kw = dict(precision=self.get('precision'), diis=int(self.get('diis')))
        if self._open_shell():
            # nAPMO's DFT takes spin 'polarized' for open shells (dft_solver.py:35)
            if nuc is None:
                drv = _scf.GridUHF(self.system, nrad, nang, charge=self._charge(),
                                   multiplicity=self._multiplicity(), exchange='lda', **kw)
            else:
                if func.get('e-:' + nuc, func.get(nuc + ':e-')):
                    raise NotImplementedError('electron-nucleus correlation with spin-polarised '
                                              'electrons is not built')
                drv = _scf.GridMultiSCF(self.system, nuc, nrad, nang, charge=self._charge(),
                                        multiplicity=self._multiplicity(), exchange='lda', **kw)
            return self._run(drv)
        if nuc is None:
            drv = _scf.GridRHF(self.system, nrad, nang, exchange='lda', **kw)
        else:
            corr = func.get('e-:' + nuc, func.get(nuc + ':e-'))
            drv = _scf.GridAPMO(self.system, nuc, nrad, nang, exchange='lda', correlation=corr,
                                **kw)
        return self._run(drv)
