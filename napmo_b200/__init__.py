"""napmo_b200: nAPMO's grid-quadrature hot path, B200-native.

Drop-in for ``napmo.grids`` / ``napmo.gto`` and the grid quadrature entry
points of ``libnapmo.so``: Becke partition weights, contracted GTOs and
gradients on grid points, rho = phi^T D phi, F = phi^T diag(w v) phi, and the
Lebedev-projected radial Poisson solve, all as sm_100a CUDA kernels behind
nAPMO's C-ABI; with nAPMO's numerical-orbital operators (``compute_kinetic``,
``compute_dpsi``, ``PSIN``, ``PSIO_BECKE``), local functionals and the
one-electron integrals of its libint interface.  Loading fails if
``lib/libnapmo.so`` has not been built.
"""
from . import cext
from .cext import NapmoError
from .grids import (AngularGrid, AtomicGrid, BeckeGrid, Cell, ChebyshevRadialTransform,
                    CubicSpline, CuspExtrapolation, Extrapolation, IndentityRadialTransform,
                    MultiGrid, PotentialExtrapolation, PowerExtrapolation,
                    PowerRadialTransform, RadialGrid, RadialTransform, ZeroExtrapolation,
                    coulomb_potential_device, lebedev_get_order, poisson_solver, solve_ode2)
from .gto import BasisSet, ContractedGaussian, PrimitiveGaussian
from .system import BOHR_TO_ANGSTROM, MolecularSystem
from .wavefunction import WaveFunction, compute_coulomb, compute_nuclear
from .fock import FockBatch, FockBuilder
from .functional import Functional, epc17_2, isc_functional_selector
from .numeric import PSIN, PSIO_BECKE, GridOperators, compute_dpsi, compute_kinetic
from .solver import DFT, HF

ANGSTROM_TO_BOHR = 1.889726133921252
