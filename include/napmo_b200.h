/*
 * napmo_b200.h -- C-ABI of libnapmo.so (napmo_b200/lib/libnapmo.so).
 *
 * Part 1 is the drop-in surface: the symbols nAPMO's Python layer binds with
 * ctypes (napmo/__init__.py:95-585, loaded by napmo/system/cext.py:11-16),
 * with the same argument order and meaning.  Each line cites the nAPMO
 * function it replaces.  Opaque handles are `void *`; arrays are plain
 * pointers to row-major doubles owned by the caller unless stated.  Entry
 * points that compute on grid points run on the current CUDA device and
 * synchronise before returning; errors are reported through
 * napmo_last_error() (nAPMO throws C++ exceptions across ctypes instead).
 *
 * Part 2 is this library's device API: device pointers, a cudaStream_t
 * passed as `void *`, int status (0 = success), no synchronisation.
 */
#ifndef NAPMO_B200_H
#define NAPMO_B200_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------- errors */
/* Last error of the calling thread: returns its code, copies the message. */
int napmo_last_error(char *buf, int len);
/* Frees arrays returned by AtomicGrid_integrate / _spherical_expansion. */
void napmo_free_array(double *p);

/* ===================================================== Part 1: drop-in */
/* ---- radial transforms: src/horton/rtransform.{h,cpp} */
void RTransform_del(void *rt);                                   /* rtransform.h:51 */
double RTransform_radius(void *rt, double t);                    /* rtransform.h:52 */
double RTransform_deriv(void *rt, double t);                     /* rtransform.h:53 */
double RTransform_deriv2(void *rt, double t);                    /* rtransform.h:54 */
double RTransform_deriv3(void *rt, double t);                    /* rtransform.h:55 */
double RTransform_inv(void *rt, double r);                       /* rtransform.h:56 */
void RTransform_radius_array(void *rt, double *t, double *r, int n);  /* rtransform.h:58 */
void RTransform_deriv_array(void *rt, double *t, double *d, int n);   /* rtransform.h:60 */
void RTransform_deriv2_array(void *rt, double *t, double *d, int n);  /* rtransform.h:62 */
void RTransform_deriv3_array(void *rt, double *t, double *d, int n);  /* rtransform.h:64 */
void RTransform_inv_array(void *rt, double *r, double *t, int n);     /* rtransform.h:66 */
int RTransform_get_npoint(void *rt);                             /* rtransform.h:67 */
void *IdentityRTransform_new(int npoint);                        /* rtransform.h:87 */
void *LinearRTransform_new(double rmin, double rmax, int npoint); /* rtransform.h:114 */
double LinearRTransform_get_rmin(void *rt);                      /* rtransform.h:115 */
double LinearRTransform_get_rmax(void *rt);                      /* rtransform.h:116 */
double LinearRTransform_get_alpha(void *rt);                     /* rtransform.h:117 */
void *ExpRTransform_new(double rmin, double rmax, int npoint);    /* rtransform.h:144 */
double ExpRTransform_get_rmin(void *rt);                         /* rtransform.h:145 */
double ExpRTransform_get_rmax(void *rt);                         /* rtransform.h:146 */
double ExpRTransform_get_alpha(void *rt);                        /* rtransform.h:147 */
void *ShiftedExpRTransform_new(double rmin, double rshift, double rmax, int npoint); /* :176 */
double ShiftedExpRTransform_get_rmin(void *rt);                  /* rtransform.h:178 */
double ShiftedExpRTransform_get_rshift(void *rt);                /* rtransform.h:179 */
double ShiftedExpRTransform_get_rmax(void *rt);                  /* rtransform.h:180 */
double ShiftedExpRTransform_get_r0(void *rt);                    /* rtransform.h:181 */
double ShiftedExpRTransform_get_alpha(void *rt);                 /* rtransform.h:182 */
void *PowerRTransform_new(double rmin, double rmax, int npoint);  /* rtransform.h:210 */
double PowerRTransform_get_rmin(void *rt);                       /* rtransform.h:211 */
double PowerRTransform_get_rmax(void *rt);                       /* rtransform.h:212 */
double PowerRTransform_get_power(void *rt);                      /* rtransform.h:213 */
void *ChebyshevRTransform_new(double radii, int npoint);         /* rtransform.h:240 */
double ChebyshevRTransform_get_radii(void *rt);                  /* rtransform.h:241 */
double ChebyshevRTransform_get_z(void *rt);                      /* rtransform.h:242 */

/* ---- angular grid: src/grid/angular.{h,cpp} (Lebedev-Laikov rules) */
void *AngularGrid_new(int lorder);                               /* angular.h:109 */
void AngularGrid_del(void *g);                                   /* angular.h:111 */
void AngularGrid_spherical(void *g);                             /* angular.h:113 */
/* GSL-based expansions (not on the grid-quadrature path): set an error. */
void AngularGrid_spherical_expansion(void *g, int lmax, int size_f, double *f,
                                     double *output);            /* angular.h:115 */
void AngularGrid_eval_expansion(void *g, int lmax, int size_f, double *dec,
                                double *output);                 /* angular.h:119 */
double AngularGrid_integrate(void *g, int segments, double *f, double *s); /* angular.h:123 */
int AngularGrid_get_lorder(void *g);                             /* angular.h:126 */
double *AngularGrid_get_points(void *g);                         /* angular.h:128 */
double *AngularGrid_get_weights(void *g);                        /* angular.h:130 */

/* ---- radial grid: src/grid/radial.{h,cpp} */
void *RadialGrid_new(void *rtf, double rad);                     /* radial.h:53 */
void RadialGrid_del(void *g);                                    /* radial.h:55 */
double RadialGrid_integrate(void *g, int segments, double *f);   /* radial.h:57 */
double *RadialGrid_deriv2(void *g, double *f);  /* radial.h:59, radial.cpp:51-192; new[] array, free with napmo_free_array */
int RadialGrid_get_size(void *g);                                /* radial.h:61 */
double RadialGrid_get_radii(void *g);                            /* radial.h:63 */
double *RadialGrid_get_points(void *g);                          /* radial.h:65 */
double *RadialGrid_get_weights(void *g);                         /* radial.h:67 */

/* ---- atomic grid: src/grid/atomic_grid.{h,cpp} */
void *AtomicGrid_new(void *angular, void *radial, double *R);    /* atomic_grid.h:73 */
void AtomicGrid_del(void *g);                                    /* atomic_grid.h:75 */
double *AtomicGrid_integrate(void *g, int nfunc, int segments, int size,
                             double *f);                         /* atomic_grid.h:77 */
double *AtomicGrid_spherical_expansion(void *g, double *f, int lmax); /* atomic_grid.h:80 (GPU) */
int AtomicGrid_get_size(void *g);                                /* atomic_grid.h:82 */
double AtomicGrid_get_radii(void *g);                            /* atomic_grid.h:84 */
double *AtomicGrid_get_origin(void *g);                          /* atomic_grid.h:86 */
double *AtomicGrid_get_points(void *g);                          /* atomic_grid.h:88 */
double *AtomicGrid_get_weights(void *g);                         /* atomic_grid.h:90 */

/* ---- Becke molecular grid: src/grid/becke.{h,cpp} (weights on the GPU) */
void *BeckeGrid_new(void **atomic_grids, int n, int l, double ld); /* becke.h:95 */
void *BeckeGrid_from_points(double *p, int sz, int nc);          /* becke.h:97 */
void BeckeGrid_del(void *g);                                     /* becke.h:99 */
double BeckeGrid_integrate(void *g, double *f);                  /* becke.h:101 (GPU) */
int BeckeGrid_get_ncenter(void *g);                              /* becke.h:103 */
int BeckeGrid_get_size(void *g);                                 /* becke.h:105 */
double *BeckeGrid_get_radii(void *g);                            /* becke.h:107 */
double *BeckeGrid_get_points(void *g);                           /* becke.h:109 */
double *BeckeGrid_get_weights(void *g);                          /* becke.h:111 */
double *BeckeGrid_get_origin(void *g);                           /* becke.h:113 */
double *BeckeGrid_get_becke_weights(void *g);                    /* becke.h:115 */

/* ---- common points between species grids: src/grid/multi_grid.{h,cpp} */
void *MultiGrid_new(int ns);                                     /* multi_grid.h:50 */
void MultiGrid_del(void *m);                                     /* multi_grid.h:52 */
int MultiGrid_add_grid(void *m, void *grid);                     /* multi_grid.h:54 */
int *MultiGrid_get_common_index(void *m, int a, int b);          /* multi_grid.h:56 (GPU) */
int MultiGrid_get_common_index_size(void *m, int a, int b);      /* multi_grid.h:59 */
int MultiGrid_get_ngrids(void *m);                               /* multi_grid.h:62 */
int MultiGrid_get_nspecies(void *m);                             /* multi_grid.h:64 */

/* ---- cell (non-periodic only): src/horton/cell.h */
void *Cell_new(double *rvecs, int nvec);                         /* cell.h:238 */
void Cell_del(void *c);                                          /* cell.h:239 */

/* ---- cubic splines and extrapolations: src/horton/{cubic_spline,extrapolation}.h */
void tridiagsym_solve(double *mid, double *up, double *right, double *sol, int n); /* cubic_spline.h:33 */
void solve_cubic_spline_system(double *y, double *dt, int npoint);   /* cubic_spline.h:35 */
void compute_cubic_spline_int_weights(double *weights, int npoint);  /* cubic_spline.h:36 */
void *CubicSpline_new(double *y, double *dt, void *ext, void *rtf, int n); /* cubic_spline.h:71 */
void CubicSpline_del(void *c);                                   /* cubic_spline.h:74 */
void CubicSpline_eval(void *c, double *x, double *y, int n);     /* cubic_spline.h:75 */
void CubicSpline_eval_deriv(void *c, double *x, double *d, int n); /* cubic_spline.h:77 */
double CubicSpline_get_first_x(void *c);                         /* cubic_spline.h:79 */
double CubicSpline_get_last_x(void *c);                          /* cubic_spline.h:80 */
void *CubicSpline_get_rtransform(void *c);                       /* cubic_spline.h:81 */
void *CubicSpline_get_extrapolation(void *c);                    /* cubic_spline.h:82 */
void Extrapolation_prepare(void *e, void *c);                    /* extrapolation.h:45 */
void Extrapolation_del(void *e);                                 /* extrapolation.h:46 */
double Extrapolation_eval_left(void *e, double x);               /* extrapolation.h:47 */
double Extrapolation_eval_right(void *e, double x);              /* extrapolation.h:48 */
double Extrapolation_deriv_left(void *e, double x);              /* extrapolation.h:49 */
double Extrapolation_deriv_right(void *e, double x);             /* extrapolation.h:50 */
bool Extrapolation_has_tail(void *e);                            /* extrapolation.h:51 */
void *ZeroExtrapolation_new(void);                               /* extrapolation.h:71 */
void *CuspExtrapolation_new(void);                               /* extrapolation.h:94 */
void *PowerExtrapolation_new(double power);                      /* extrapolation.h:164 */
double PowerExtrapolation_get_power(void *e);                    /* extrapolation.h:165 */
void *PotentialExtrapolation_new(int l);                         /* extrapolation.h:167 */

/* ---- Hermite finite elements and moments: src/horton/{ode2,dot_multi,moments,evaluate}.h */
double hermite_overlap2(long xmax, long i0, bool d0, long i1, bool d1);  /* ode2.h:27 */
double hermite_overlap3(long xmax, long i0, bool d0, long i1, bool d1, long i2,
                        bool d2);                                /* ode2.h:28 */
void build_ode2(double *b, double *a, double *f, double *bcs, double *coeffs, double *rhs,
                long npoint);                                    /* ode2.h:37 */
void fill_pure_polynomials(double *output, long lmax);           /* moments.h (moments.cpp:59) */
void dot_multi_moments(long npoint, long nvector, double *data, double *points,
                       double *center, long lmax, long mtype, long *segments,
                       double *output, long nmoment);            /* dot_multi.h:37 (GPU) */
void eval_decomposition_grid(void **splines, double *center, double *output, double *points,
                             void *cell, long nspline, long npoint); /* evaluate.h:43 (GPU) */

/* ---- Gaussian basis: src/system/{gto,basis_set}.h */
void *PrimitiveGaussian_new(int *l, double *A, double zeta, double coeff); /* gto.h:112 */
void PrimitiveGaussian_del(void *p);
void PrimitiveGaussian_get_l(void *p, int *l);                   /* gto.h:115 */
void PrimitiveGaussian_get_origin(void *p, double *A);           /* gto.h:117 */
void PrimitiveGaussian_compute(void *p, double *r, double *out, int size); /* gto.h:119 (GPU) */
void PrimitiveGaussian_deriv(void *p, double *r, double *out, int size);   /* gto.h:122 (GPU) */
double PrimitiveGaussian_overlap(void *p, void *q);              /* gto.h:125 */
double PrimitiveGaussian_get_zeta(void *p);                      /* gto.h:127 */
double PrimitiveGaussian_get_coeff(void *p);                     /* gto.h:129 */
double PrimitiveGaussian_get_norma(void *p);                     /* gto.h:131 */
void *ContractedGaussian_new(void **prims, int n);               /* gto.h:200 */
void ContractedGaussian_del(void *c);
int ContractedGaussian_get_nprim(void *c);                       /* gto.h:203 */
void ContractedGaussian_get_l(void *c, int *l);                  /* gto.h:205 */
void ContractedGaussian_get_origin(void *c, double *A);          /* gto.h:207 */
void ContractedGaussian_compute(void *c, double *r, double *out, int size); /* gto.h:209 (GPU) */
void ContractedGaussian_deriv(void *c, double *r, double *out, int size);   /* gto.h:212 (GPU) */
double ContractedGaussian_overlap(void *c, void *o);             /* gto.h:215 */
double ContractedGaussian_get_norma(void *c);                    /* gto.h:218 */
void *BasisSet_new_empty(void);                                  /* basis_set.h:53 */
void *BasisSet_new(void **contractions, int n);                  /* basis_set.h:55 */
void BasisSet_del(void *b);
void BasisSet_compute(void *b, double *r, double *out, int size); /* basis_set.h:57 (GPU) */
void BasisSet_deriv(void *b, double *r, double *out, int size);   /* basis_set.h:59 (GPU) */
void BasisSet_update(void *b, void *other);                      /* basis_set.h:61 */
int BasisSet_get_nbasis(void *b);                                /* basis_set.h:63 */
int BasisSet_get_max_l(void *b);                                 /* basis_set.h:65 */
int BasisSet_get_max_nprim(void *b);                             /* basis_set.h:67 */

/* ---- wave function (struct wf, src/wavefunction/wavefunction.h:20-44) */
void wavefunction_guess_hcore(void *psi);                        /* wavefunction.h:51 */
void wavefunction_transformation_matrix(void *psi);              /* wavefunction.h:53 */
void wavefunction_compute_coefficients(void *psi);               /* wavefunction.h:55 */
void wavefunction_compute_density(void *psi);                    /* wavefunction.h:57 */
void wavefunction_compute_energy(void *psi);                     /* wavefunction.h:59 */
void wavefunction_iterate(void *psi);                            /* wavefunction.h:61 */
void nwavefunction_compute_density_from_dm(void *basis, void *grid, double *dm,
                                           double *output, double epsilon,
                                           double *dmmaxrow);    /* wavefunction.h:70 (GPU) */
void nwavefunction_compute_2body_matrix(void *psi, void *grid, double *phi, double *J,
                                        double *K);              /* wavefunction.h:74 (GPU) */
void nwavefunction_compute_coupling(void *psi, void *grid, double *phi, double *other_J,
                                    double *res);                /* wavefunction.h:77 (GPU) */
void nwavefunction_compute_xc_matrix(void *psi, void *grid, double *phi,
                                     double *xc_vrho);           /* wavefunction.h:80 (GPU) */

/* ---- analytic integrals / auxiliary basis (libint2, not on the grid
 * path): present so the ctypes layer binds, every call sets an error.
 * src/ints/libint_iface.h:106-148, src/grid/auxiliary_basis.h */
/* One-body part of nAPMO's libint interface (libint_iface.cpp:41-190, 1318-1345),
 * computed on the device (ints.cu): add the species' bases and point charges, then
 * kind 1 = overlap, 2 = kinetic, 3 = nuclear attraction -sum Z <1/r_C> into a host
 * [n][n] matrix of unit-normalised contracted functions. */
void *LibintInterface_new(int id);
void LibintInterface_del(void *l);
void LibintInterface_add_basis(void *l, void *b);
void LibintInterface_add_pointcharges(void *l, int z, double *center);
int LibintInterface_get_nbasis(void *l);
void LibintInterface_compute_1body_ints(void *l, int kind, double *out);
void LibintInterface_init_2body_ints(void *l);
void *LibintInterface_compute_2body_ints(void *l, double *D);
void LibintInterface_compute_2body_direct(void *l, double *D, double *G);
void LibintInterface_compute_coupling_direct(void *l, void *o, double *D, double *J);
void *LibintInterface_diis_new(int n);
void LibintInterface_diis(void *d, void *psi);
void wavefunction_compute_2body_matrix(void *psi, void *ints);
void *AuxiliaryBasis_new(void *grid);
void AuxiliaryBasis_del(void *a);
double *AuxiliaryBasis_get_aobasis(void *a);
int AuxiliaryBasis_get_nao(void *a);

/* ================================================== Part 2: device API */
/* Device pointers of a grid's mirror: points (SoA), weights, Becke weights. */
/* Moves the grid's centres (origin [ncenter][3], bohr): points rebuilt as at
 * construction (atomic_grid.cpp:12-51), device mirror rewritten in place,
 * Becke weights recomputed, Poisson tables dropped.  No counterpart in nAPMO
 * (it builds a new grid per geometry). */
int napmo_grid_set_centers(void *grid, const double *origin);
int napmo_grid_device_arrays(void *grid, double **x, double **y, double **z, double **w,
                             double **wb);
/* Becke weights of device points (SoA) owned by atoms through atom_offset
 * (host, ncenter+1); replaces BeckeGrid::compute_weights, becke.cpp:79-176. */
int napmo_gpu_becke_weights(int npoint, int ncenter, const double *x, const double *y,
                            const double *z, const double *origin, const double *radii,
                            const int *atom_offset, double *out, void *stream);
/* phi[mu * ld + p] (and gradients grad[(c * nbasis + mu) * ld + p]) at device
 * points; replaces BasisSet_compute / BasisSet_deriv (basis_set.cpp:69-99). */
int napmo_gpu_basis_values(void *basis, int npoint, const double *x, const double *y,
                           const double *z, double *phi, long ld, double *grad, void *stream);
/* rho[p] = sum D[mu][nu] phi[mu][p] phi[nu][p]; phi [n][ld], ld >= npoint
 * rounded up to 128, zero padded; replaces the density of psi_hybrid.py:144-150. */
int napmo_gpu_density(int n, int npoint, const double *phi, long ld, const double *D,
                      double *rho, void *stream);
/* F = phi diag(wv) psi^T (psi = phi if null), upper triangle mirrored;
 * replaces nwavefunction_compute_coupling/_xc_matrix (nwavefunction.cpp:77-197).
 * phi, psi [n][ld] and wv are 16-byte aligned, ld even and >= npoint rounded up
 * to 128, every array zero padded to that length; npoint = 0 gives F = 0. */
int napmo_gpu_quadrature(int n, int npoint, const double *phi, const double *psi, long ld,
                         const double *wv, double *F, void *stream);
/* wv = wb w (q v + vext), zero padded to the next multiple of 128. */
int napmo_gpu_combine_weights(int npoint, const double *wb, const double *w, double q,
                              const double *v, const double *vext, double *wv, void *stream);
/* Coulomb potential of rho on the grid's points (projection, radial FEM
 * solves, multipole evaluation); replaces compute_coulomb / poisson_solver
 * (ntwobody.py:15-46, poisson_solver.py:18-118, evaluate.cpp:129-220). */
int napmo_gpu_poisson(void *grid, const double *rho, int lmax, double *v, int accumulate,
                      double *raw_y, double *raw_dt, void *stream);
long napmo_poisson_raw_size(void *grid, int lmax);
/* k solves in one call: v[j] = V_H[rho[j]], device rows of ld >= grid size (the
 * orbital-pair densities of exchange, psi_numeric.py:186-215). */
int napmo_gpu_poisson_many(void *grid, int k, const double *rho, long ld, int lmax, double *v,
                           void *stream);
/* Truncation tolerance (a.u.) of the grid's potential evaluation.  No
 * counterpart in nAPMO, whose evaluate.cpp:129-220 sums every (l, m) <= lmax:
 * 0 (the default) does the same; tol > 0 lets each (atom, radial interval)
 * drop its highest l-blocks while their bounded sum stays <= tol, so each
 * point's potential moves by at most natom * tol. */
int napmo_grid_set_poisson_tolerance(void *grid, double tol);
/* LDA exchange (Dirac-Slater) and VWN5 correlation of rho (device, n values):
 * energies per particle and potentials, any output may be null; replaces
 * Functional('lda').compute_exchange / compute_correlation
 * (napmo/functional/xc_interface.py:62-90, LibXC lda_x / lda_c_vwn). */
int napmo_gpu_lda_xc(long n, const double *rho, double *x_zk, double *x_vrho, double *c_zk,
                     double *c_vrho, void *stream);
/* Spin-polarised LDA exchange and VWN5 correlation of (rho_a, rho_b) (device,
 * n values each): energies per particle of the total density and both spins'
 * potentials, any output may be null; replaces Functional('lda') with spin
 * 'polarized' (xc_interface.py:62-90, LibXC lda_x / lda_c_vwn), which nAPMO's
 * DFT uses for open shells (dft_solver.py:35).  nAPMO interleaves the spins in
 * one array; here they are two. */
int napmo_gpu_lda_xc_polarized(long n, const double *rho_a, const double *rho_b, double *x_zk,
                               double *x_va, double *x_vb, double *c_zk, double *c_va,
                               double *c_vb, void *stream);
/* epc17-2 electron-proton correlation at n common points (device): energy per
 * electron and both species' potentials; replaces epc17_2
 * (napmo/functional/interspecies_correlation.py:36-68). */
int napmo_gpu_epc17_2(long n, const double *rho_e, const double *rho_n, double *ene,
                      double *pot_e, double *pot_n, void *stream);
/* Numerical-orbital operators on the grid (device rows of ld >= grid size).
 * Kinetic: out[k] = scale * (-1/2 laplacian psi[k]); replaces compute_kinetic
 * (napmo/wavefunction/nkinetic.py:15-73, RadialGrid::deriv2 of
 * src/grid/radial.cpp:51-192).  Chebyshev radial grids of >= 8 points. */
int napmo_gpu_kinetic(void *grid, int lmax, int nfunc, const double *psi, long ld, double scale,
                      double *out, void *stream);
/* Becke-Dickson orbital corrections of nfunc orbitals; replaces compute_dpsi
 * (napmo/wavefunction/ndpsi.py:15-89).  doi, oi: host arrays of nfunc.  The
 * workspace lives on the grid's Poisson tables: calls on one grid (and its
 * Poisson solves) must not overlap on the device. */
int napmo_gpu_dpsi(void *grid, int lmax, int nfunc, const double *phi, const double *resid,
                   const double *vtot, long ld, const double *doi, const double *oi,
                   double mass_inv, double *out, void *stream);
/* M[i][j] = integral A_i B_j over the grid (n x m, device); replaces
 * get_operator_matrix (napmo/wavefunction/psi_numeric.py:406-424). */
int napmo_gpu_operator_matrix(void *grid, int n, int m, const double *A, long lda,
                              const double *B, long ldb, double *M, void *stream);
/* S, T, V = -sum_C Z_C <mu|1/r_C|nu> of a basis (device [n][n] outputs, any may be
 * null; charges host [nq][4] = x, y, z, Z); replaces libint's one-body engines
 * (libint_iface.cpp:136-190) and overlap.cpp:12-64. */
int napmo_gpu_one_body(void *basis, int nq, const double *charges, double *S, double *T,
                       double *V, void *stream);
/* sum_A Z_A / |r - R_A| at device points; replaces compute_nuclear (nnuclear.py:15-37). */
int napmo_gpu_nuclear_potential(int npoint, const double *x, const double *y, const double *z,
                                int nq, const double *charges, double *v, void *stream);

/* Allocation-free twin of napmo_gpu_quadrature for callers that cannot
 * allocate device memory while calling the library (hosts that budget all GPU
 * memory themselves; callers that must not let an allocation stall the
 * device).  No counterpart in nAPMO.  Split-K scratch is a fixed 16 MiB device
 * array inside the library (held by every GPU that loads it until exit), so
 * n <= 1920; larger n is refused with an error.  Each call looks up the
 * array's device address (no allocation); the first call on a device may load
 * the library's device code, so make it before any stream capture.  Inputs as
 * for napmo_gpu_quadrature: phi, psi, wv 16-byte aligned, ld even and >=
 * npoint rounded up to 128, wv zero padded to that length (as
 * napmo_gpu_combine_weights writes it); npoint = 0 gives F = 0.  Calls share
 * the array: overlapping calls on the GPU race. */
int napmo_gpu_quadrature_noalloc(int n, int npoint, const double *phi, const double *psi,
                                 long ld, const double *wv, double *F, void *stream);

/* Fock-build plan: phi of `basis` on `grid` evaluated once and kept in HBM
 * with the Poisson tables of `lmax`; per build rho -> V_H -> F (the chain of
 * psi_hybrid.py:81-110 / psi_numeric.py:152-241).  lmax >= 0: one cutoff for
 * all atoms (nAPMO: lebedev_get_order(nang) // 2, psi_numeric.py:66); -1: no
 * Poisson tables (quadratures only); -2: per atom, from its own Lebedev rule
 * (grids with different angular sizes per atom). */
void *napmo_fock_plan_new(void *grid, void *basis, int lmax, void *stream);
void napmo_fock_plan_free(void *plan);
/* Re-evaluates the plan's basis values after its grid or basis moved, in its
 * own buffers; rebuilds the int8 images and Poisson tables it holds.  No
 * counterpart in nAPMO (new objects per geometry). */
int napmo_fock_plan_refresh(void *plan, void *stream);
/* Sizes and the device phi [n][ld]; evaluates phi again first when
 * napmo_fock_plan_release_phi freed it (synchronises then). */
int napmo_fock_plan_info(void *plan, int *n, int *npoint, long *ld, double **phi);
int napmo_fock_plan_density(void *plan, const double *D, double *rho, void *stream);
int napmo_fock_plan_quadrature(void *plan, double q, const double *v, const double *vext,
                               double *F, void *stream);
int napmo_fock_plan_build(void *plan, const double *D, double q, const double *vext, double *F,
                          double *rho_out, double *v_out, void *stream);
/* v = V_H[rho] on the plan's grid with the plan's lmax and Poisson tolerance;
 * replaces compute_coulomb (ntwobody.py:15-46) inside an SCF iteration. */
int napmo_fock_plan_poisson(void *plan, const double *rho, double *v, void *stream);
/* k such solves in one call on device rows of ld >= npoint doubles. */
int napmo_fock_plan_poisson_many(void *plan, int k, const double *rho, long ld, double *v,
                                 void *stream);
/* Host-buffer twin of napmo_fock_plan_build (copies inside the call). */
int napmo_fock_plan_build_host(void *plan, const double *D, double q, const double *vext,
                               double *F, void *stream);
/* Precision of a plan's contractions: 0 FP64 (default), 1 int8 slices on the
 * tensor cores (tcgen05 kind::i8: four balanced base-256 digits per value
 * against a group exponent, exact int32 accumulation).  No counterpart in
 * nAPMO (its quadratures are FP64 only, src/wavefunction/nwavefunction.cpp). */
int napmo_fock_plan_set_precision(void *plan, int mode);
/* Truncation tolerance (a.u.) of the plan's Poisson potential evaluation: per
 * (atom, radial interval), the highest l-blocks whose bounded contribution
 * sums to at most tol are skipped.  No counterpart in nAPMO (evaluate.cpp:
 * 129-220 sums every (l, m)).  set_precision resets it: 0 for mode 0 (every
 * (l, m), as nAPMO), 1e-9 for mode 1. */
int napmo_fock_plan_set_poisson_tolerance(void *plan, double tol);
/* Point screening of the plan's current mode (mode 1 keeps the points with
 * |w_becke w| max_mu phi_mu(p)^2 >= 1e-24; rho and v are 0 at the others).
 * *keep: device flags, one int per grid point (null when all points are used);
 * *nkeep: kept points.  No counterpart in nAPMO (every point is used). */
int napmo_fock_plan_screening(void *plan, const int **keep, int *nkeep);
/* Point screening of the FP64 mode (precision 1 always screens): tol > 0
 * keeps the points with |wb w| max_mu phi_mu(p)^2 >= tol (1e-24 is the int8
 * mode's threshold) for the density, the potential evaluation and the
 * quadrature; 0 restores every point (nAPMO's sums).  No counterpart in nAPMO.
 * Synchronises. */
int napmo_fock_plan_set_fp64_screening(void *plan, double tol, void *stream);
/* Device bytes of the plan's int8 operand images and scratch. */
long napmo_fock_plan_int8_bytes(void *plan);
/* Precision 1 only: frees the plan's FP64 phi (n x ld doubles), which the
 * int8 builds do not read; whatever needs it again (an FP64 build,
 * napmo_fock_plan_info, set_fp64_screening, a switch back to precision 0,
 * refresh) evaluates it again first.  No counterpart in nAPMO.
 * Synchronises. */
int napmo_fock_plan_release_phi(void *plan);
/* Batched Fock builds of many plans (molecules of uneven size) by one CUDA
 * graph launch; no counterpart in nAPMO (its SCF drivers loop over species,
 * scf.py:146-273).  The batch owns a device D and F per plan
 * (napmo_fock_batch_buffers); napmo_fock_batch_build captures the builds on
 * first use (after one eager warm-up) and then launches the graph on `stream`.
 * napmo_fock_batch_tune times candidate launch shapes (capture streams x
 * CTA budget of the int8 kernels) and keeps the fastest. */
void *napmo_fock_batch_new(void **plans, int nplan, double q);
void napmo_fock_batch_free(void *batch);
int napmo_fock_batch_buffers(void *batch, int i, double **D, double **F);
int napmo_fock_batch_build(void *batch, void *stream);
int napmo_fock_batch_tune(void *batch, void *stream, int reps, int *nstream, int *budget,
                          double *ms);
int napmo_fock_batch_config(void *batch, int *nstream, int *budget);
/* Build mode of a batch: 0 = the molecules' own launch chains over capture
 * streams (default); 1 = one launch per stage for the whole batch: persistent
 * density and quadrature launches taking (molecule, tile) items from device
 * work queues (bounded waits), one Poisson plan over all the molecules' grids.
 * No counterpart in nAPMO (its builds are per molecule, psi_hybrid.py:81-110). */
int napmo_fock_batch_set_mode(void *batch, int mode);
/* Mode 1: runs the density stage with a work queue that is never posted, so
 * that every wait runs out after timeout_s (<= 10 s); *status = 5 then.  A test
 * of the bounded waits without a fault; the batch stays usable. */
int napmo_fock_batch_queue_selftest(void *batch, double timeout_s, void *stream, int *status);
/* Mode 1: error word of the work queues since the last call (0, or 5 when a
 * wait ran out); clears it. */
int napmo_fock_batch_status(void *batch, void *stream, int *status);

/* Grid quadrature energy of one species in a point-charge potential and its
 * nuclear-coordinate gradient (Becke weights, basis functions, grid points and
 * charges all differentiated): E = sum_p wq wb rho_D v, v = sum_C q_C/|r-R_C|.
 * D device [n][n]; charges host [nq][4] = x, y, z, q; outputs host: E,
 * grad[ncenter][3] (grid centres, which carry the points and the basis
 * shells), grad_q[nq][3] (charge positions).  dE/dD is the quadrature matrix
 * of wq wb v (napmo_fock_plan_quadrature with vext = v).  No counterpart in
 * nAPMO; up to 16 centres, 16 charges, 192 basis functions. */
int napmo_grid_energy_gradient(void *grid, void *basis, const double *D, int nq,
                               const double *charges, double *E, double *grad, double *grad_q,
                               void *stream);

/* Analytic overlap and kinetic-energy matrices (host, [n][n]) of a basis
 * (Obara-Saika); nAPMO obtains them from libint (libint_iface.cpp:136-190). */
int napmo_basis_one_body(void *basis, double *S, double *T);
/* Origins [nfunc][3] of the basis functions; moving them (functions of one
 * shell together) rewrites the device shell centres in place.  No
 * counterpart in nAPMO (its basis is rebuilt per geometry). */
int napmo_basis_get_origins(void *basis, double *out);
int napmo_basis_set_origins(void *basis, const double *origins);

/* Error word of the tensor-core kernels (0 none, 5 an mbarrier wait ran out);
 * synchronises the stream, `reset` nonzero clears it. */
int napmo_tc_status(void *stream, int reset);
/* Runs the tensor-core kernels' bounded mbarrier wait on barriers nothing
 * arrives on (about 2 s): out_dev[0..1] (device ints) receive 0 when both
 * waiting roles gave up; napmo_tc_status then reads 5.  A test of the timeout
 * path without a fault; no counterpart in nAPMO. */
int napmo_tc_wait_selftest(int *out_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NAPMO_B200_H */
