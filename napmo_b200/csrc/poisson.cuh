// Device-side Becke-Dickson Poisson solver (A. D. Becke, R. M. Dickson,
// J. Chem. Phys. 89, 2993 (1988)) as used by nAPMO's grid Coulomb potential
// (napmo/grids/poisson_solver.py:18-118, napmo/utilities/ode2.py:35-118,
// napmo/wavefunction/ntwobody.py:15-46, src/horton/evaluate.cpp:129-220).
#pragma once

#include <cuda_runtime.h>

#include "device_types.h"

namespace napmo {

// Per-atom metadata of a (possibly batched) Poisson problem.
struct PoissonAtom {
  double cx, cy, cz;
  double first_x, last_x;  // radius of the first / last radial point
  RTParams rt;
  int point_off;  // first grid point of this atom
  int nrad, nang, lmax;
  int rad_off;    // radial tables: 8 arrays of nrad (see kRad*)
  int ytab_off;   // [nang][lsize] solid harmonics of the Lebedev directions
  int proj_off;   // [nrad][lsize] projected density
  int spl_off;    // [nrad-1][lsize][4] cubic coefficients (scaled)
  int amp_off;    // [lsize][2] left / right extrapolation amplitudes (scaled)
  int raw_off;    // [lsize][nrad] solution values y and t-derivatives dt
  int mol_point_start, mol_npoint;  // points of this atom's molecule
  int bucket_off;  // [nrad + 1] buckets: 0 left tail, 1 + j interval j, nrad right tail
  int sys_off;     // radial system of (this atom, l) = sys_off + l
  long pair_off;   // this atom's slice of the (atom, point) pair arrays
  long scr_off;    // radial-solve scratch: [3 nrad][lsize]
};

// One CTA of the bucketed evaluation: `count` (<= the plan's chunk) pairs of one
// atom that share one spline interval (or tail) of that atom.
struct EvalItem {
  int atom, bucket, start, count;
};
constexpr int kEvalChunk = 128;     // default pairs per item
constexpr int kEvalChunkMax = 512;  // largest item (PoissonDev::eval_chunk)
constexpr int kEvalPerThread = 2;   // pairs evaluated by one thread

// Radial table slots (each nrad long, at rad_off + slot * nrad).
enum : int {
  kRadR = 0,      // radius
  kRadW = 1,      // radial weight 4 pi r^2 dr/dt
  kRadJ1 = 2,     // dr/dt
  kRadJ2 = 3,     // d2r/dt2
  kRadJ3 = 4,     // d3r/dt3
  kRadSigma = 5,  // sum of the atomic weights of the shell
  kRadDen = 6,    // Thomas-algorithm denominators of the spline system
  kRadUp = 7,     // Thomas-algorithm modified super-diagonal
  kRadSlots = 8,
};

// Band of the 2n x 2n radial FEM matrix: kl = ku = 3; fill-in from partial
// pivoting reaches kl + ku above the diagonal, kW stored diagonals.
constexpr int kKL = 3, kKU = 3, kW = 2 * kKL + kKU + 1;

struct PoissonDev {
  int natom = 0, nmol = 0, nsys = 0;
  int max_lmax = 0, max_nrad = 0, max_nang = 0;
  PoissonAtom *atoms = nullptr;
  int *mol_atom_off = nullptr;   // nmol + 1
  int *mol_point_off = nullptr;  // nmol + 1
  int *sys_atom = nullptr;       // radial systems (atom, l)
  int *sys_l = nullptr;
  double *rad = nullptr;
  double *ytab = nullptr;
  double *proj = nullptr;
  double *spl = nullptr;
  double *amp = nullptr;
  double *raw_y = nullptr;
  double *raw_dt = nullptr;
  // LU factors of the radial FEM systems (built once per grid): per system
  // the band [2 nrad][kW], multipliers [2 nrad][3], pivots [2 nrad]; strides
  // use lu_stride = 2 max_nrad rows
  double *lu = nullptr;
  double *lmul = nullptr;
  int *lpiv = nullptr;
  int lu_stride = 0;
  // radial-solve scratch per column (spline t-derivatives, eliminated
  // right-hand side); one solve's scratch is rscr_stride doubles long
  double *rscr = nullptr;
  long rscr_stride = 0;
  // projection scratch: rho wb w at every grid point (one solve's is
  // pg_stride doubles long)
  double *pg = nullptr;
  long pg_stride = 0;
  // bucketed evaluation (built once per grid): for every atom the points of
  // its molecule sorted by spline interval, and a partial potential per pair
  long npair = 0;
  int nitems = 0;
  int nitems_inner = 0;        // items [0, nitems_inner) lie inside their atom's grid
  int eval_chunk = kEvalChunk;  // pairs per item (<= kEvalChunkMax); CTA = chunk / 2 threads
  int *pairs = nullptr;        // point index, bucket-sorted per atom
  double2 *pair_u = nullptr;   // (u, 1/d) of each interior pair (slot order)
  EvalItem *items = nullptr;
  double *pair_v = nullptr;    // [atom][molecule point] contribution
  // Truncation of the bucketed evaluation: with lcut null every (l, m) <=
  // lmax is evaluated, as the reference does; with lcut set (one int per
  // bucket) each bucket drops its highest l-blocks whose bounded contribution
  // to any pair's potential sums to at most eval_tol (a.u.).
  double eval_tol = 0.0;
  int *lcut = nullptr;
  // Point screening: with keep set, only points with keep[p] != 0 have pairs
  // (the pair lists were built with the same flags) and the others get v = 0.
  const int *keep = nullptr;
  // Batched solves: nbatch densities batch_ld points apart, solved by the same
  // launches (project, radial, evaluate); each solve's tables lie *_stride
  // doubles (ints for lcut) apart.  nbatch = 1: one solve, strides unused.
  int nbatch = 1;
  long batch_ld = 0;
  long proj_stride = 0, spl_stride = 0, amp_stride = 0, lcut_stride = 0, pairv_stride = 0;
};

// Radial stage of the pipeline.  The default is the Poisson equation
// (u'' + 2/r u' - l(l+1)/r^2 u = -4 pi f_lm, Dirichlet values from the radial
// moments).  With `vsph` set it is the Becke-Dickson orbital correction of
// napmo/wavefunction/ndpsi.py:15-89: u'' + 2/r u' + a u = fscale f_lm with
// a = ascale (l(l+1)/r^2 + (vsph - e) - de), u = 0 at both ends.
struct RadialOp {
  double fscale = -4.0 * 3.14159265358979323846;  // source factor
  const double *vsph = nullptr;  // per shell, at atom offset rad_off / kRadSlots
  double ascale = 0.0;           // -2 / mass_inv
  double e = 0.0, de = 0.0;      // orbital energy and its correction
  bool zero_bc = false;          // u = 0 at the first and last radial point
};

// Uploads the Hermite FEM integral tables and solid-harmonic norms to
// constant memory (idempotent, per device).
cudaError_t poisson_init_constants();

// rho -> projected density (rho * wb * w projected on S_lm per shell).
cudaError_t launch_poisson_project(const PoissonDev &P, const double *rho,
                                   const double *wb, const double *w,
                                   cudaStream_t s);
// Assembles and LU-factors the radial FEM matrices (once per grid).
cudaError_t launch_poisson_factor(const PoissonDev &P, cudaStream_t s);
// projected density -> spline tables of the potential (one thread per (solve,
// l, m) column, one CTA per (atom, l) and group of solves); needs P.rscr.
cudaError_t launch_poisson_radial(const PoissonDev &P, cudaStream_t s);
// The same two stages for another radial operator (factors into P.lu, P.lmul,
// P.lpiv; raw spline output skipped when P.raw_y is null).
cudaError_t launch_radial_factor(const PoissonDev &P, const RadialOp &op, cudaStream_t s);
cudaError_t launch_radial_solve(const PoissonDev &P, const RadialOp &op, cudaStream_t s);
// Kinetic operator of nAPMO's numerical orbitals (nkinetic.py:15-73):
// projected function -> spline tables of scale * (1/r d2/dr2 r - l(l+1)/r^2)
// f_lm (radial second derivative by finite differences in the Chebyshev angle,
// src/grid/radial.cpp:51-192).  Every atom must use the Chebyshev transform
// and >= 8 radial points.
cudaError_t launch_kinetic_radial(const PoissonDev &P, double scale, cudaStream_t s);
// Per atom and radial shell: sum_j f wb w / sum_j w over the shell's
// directions (AtomicGrid.spherical_average of f wb); out at rad_off / kRadSlots.
cudaError_t launch_shell_average(const PoissonDev &P, const double *f, const double *wb,
                                 const double *w, double *out, cudaStream_t s);
// Pair-list construction: bucket of every (atom, point) pair and the bucket
// populations (count[atom.bucket_off + b], atomics on integers), then the
// bucket-sorted point lists (order inside a bucket is irrelevant: each pair
// writes its own slot of pair_v).
// With keep non-null, points whose flag is 0 get no pair (bucket -1).
cudaError_t launch_pair_buckets(const PoissonDev &P, int max_mol_npoint, const double *x,
                                const double *y, const double *z, const int *keep,
                                int *bucket_of, int *count, cudaStream_t s);
// The scatter also stores, for the pairs of interior buckets, the spline
// interval coordinate u = rt_inv(|p - A|) - j and 1 / |p - A| in P.pair_u
// (slot order).
cudaError_t launch_pair_scatter(const PoissonDev &P, int max_mol_npoint, const double *x,
                                const double *y, const double *z, const int *bucket_of,
                                int *cursor, cudaStream_t s);
// spline tables -> potential at every grid point (out = or += ).  Uses the
// bucketed pair lists when P.items is set, the point-parallel kernel otherwise.
cudaError_t launch_poisson_evaluate(const PoissonDev &P, int npoint,
                                    const double *x, const double *y,
                                    const double *z, double *out, bool accumulate,
                                    cudaStream_t s);

}  // namespace napmo
