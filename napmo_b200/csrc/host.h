// Host-side objects behind the nAPMO-compatible C-ABI: radial transforms,
// Lebedev rules, radial/angular/atomic/Becke grids, Cartesian GTO basis sets,
// cubic splines with their extrapolations, and the Hermite finite-element
// matrix of the radial Poisson ODE.
//
// Grid construction stays on the host in FP64 and follows nAPMO's operation
// order exactly, so points and quadrature weights are bit-identical to the
// reference (src/grid/{radial,angular,atomic_grid,becke}.cpp,
// src/horton/rtransform.cpp).  Everything evaluated per grid point (Becke
// weights, basis functions, densities, quadratures, the Poisson pipeline)
// runs in the CUDA kernels of this package.
#pragma once

#include <cmath>
#include <vector>

#include "device_types.h"

namespace napmo {

// ---------------------------------------------------------------- transforms
// r = f(t) on the uniform t-axis 0..npoint-1 (src/horton/rtransform.cpp).
struct RTransform {
  int npoint;
  explicit RTransform(int n) : npoint(n) {}
  virtual ~RTransform() {}
  virtual double radius(double t) const = 0;
  virtual double deriv(double t) const = 0;
  virtual double deriv2(double t) const = 0;
  virtual double deriv3(double t) const = 0;
  virtual double inv(double r) const = 0;
  virtual RTParams params() const = 0;
};

struct IdentityRT : RTransform {
  explicit IdentityRT(int n) : RTransform(n) {}
  double radius(double t) const override { return t; }
  double deriv(double) const override { return 1.0; }
  double deriv2(double) const override { return 0.0; }
  double deriv3(double) const override { return 0.0; }
  double inv(double r) const override { return r; }
  RTParams params() const override;
};

struct LinearRT : RTransform {
  double rmin, rmax, alpha;
  LinearRT(double a, double b, int n);
  double radius(double t) const override { return alpha * t + rmin; }
  double deriv(double) const override { return alpha; }
  double deriv2(double) const override { return 0.0; }
  double deriv3(double) const override { return 0.0; }
  double inv(double r) const override { return (r - rmin) / alpha; }
  RTParams params() const override;
};

struct ExpRT : RTransform {
  double rmin, rmax, alpha;
  ExpRT(double a, double b, int n);
  double radius(double t) const override { return rmin * exp(t * alpha); }
  double deriv(double t) const override { return rmin * alpha * exp(t * alpha); }
  double deriv2(double t) const override {
    return rmin * alpha * alpha * exp(t * alpha);
  }
  double deriv3(double t) const override {
    return rmin * alpha * alpha * alpha * exp(t * alpha);
  }
  double inv(double r) const override { return log(r / rmin) / alpha; }
  RTParams params() const override;
};

struct ShiftedExpRT : RTransform {
  double rmin, rshift, rmax, r0, alpha;
  ShiftedExpRT(double a, double s, double b, int n);
  double radius(double t) const override { return r0 * exp(t * alpha) - rshift; }
  double deriv(double t) const override { return r0 * alpha * exp(t * alpha); }
  double deriv2(double t) const override {
    return r0 * alpha * alpha * exp(t * alpha);
  }
  double deriv3(double t) const override {
    return r0 * alpha * alpha * alpha * exp(t * alpha);
  }
  double inv(double r) const override { return log((r + rshift) / r0) / alpha; }
  RTParams params() const override;
};

struct PowerRT : RTransform {
  double rmin, rmax, power;
  PowerRT(double a, double b, int n);
  double radius(double t) const override { return rmin * pow(t + 1, power); }
  double deriv(double t) const override {
    return power * rmin * pow(t + 1, power - 1);
  }
  double deriv2(double t) const override {
    return power * (power - 1) * rmin * pow(t + 1, power - 2);
  }
  double deriv3(double t) const override {
    return power * (power - 1) * (power - 2) * rmin * pow(t + 1, power - 3);
  }
  double inv(double r) const override { return pow(r / rmin, 1.0 / power) - 1; }
  RTParams params() const override;
};

// Becke's map r = r_m (1 + x) / (1 - x), x = cos(pi (N - t) / (N + 1)).
struct ChebyshevRT : RTransform {
  double radii, z;
  ChebyshevRT(double rm, int n) : RTransform(n), radii(rm), z(M_PI / (n + 1)) {}
  double radius(double t) const override {
    t = npoint - t;
    double aux = cos(t * z);
    return radii * (1 + aux) / (1 - aux);
  }
  double deriv(double t) const override {
    t = npoint - t;
    double aux = t * z;
    return (2 * radii * z * sin(aux)) / pow(cos(aux) - 1, 2);
  }
  double deriv2(double t) const override {
    t = npoint - t;
    double aux = t * z;
    return 0.5 * z * z * radii * (2 + cos(aux)) * pow(1 / sin(aux * 0.5), 4);
  }
  double deriv3(double t) const override {
    t = npoint - t;
    double aux = t * z;
    double half = aux * 0.5;
    return 0.25 * z * z * z * radii * (11 * cos(half) + cos(1.5 * aux)) *
           pow(1 / sin(half), 5);
  }
  double inv(double r) const override {
    return -(acos((r - radii) / (r + radii)) / z) + npoint;
  }
  RTParams params() const override;
};

// ------------------------------------------------------------------- Lebedev
// Fills x, y, z, w (each `order` long).  Returns false for unknown orders.
bool lebedev_rule(int order, double *x, double *y, double *z, double *w);
int lebedev_precision(int order);  // -1 for unknown orders

// --------------------------------------------------------------------- grids
struct RadialGrid {
  RTransform *rtf;  // not owned
  double radii;
  std::vector<double> points, weights;
  RadialGrid(RTransform *rt, double rad);
  double integrate(int segments, const double *f) const;
};

struct AngularGrid {
  int lorder;
  std::vector<double> points;  // [lorder][3]
  std::vector<double> weights;
  explicit AngularGrid(int order);
};

struct AtomicGrid {
  AngularGrid *ang;  // not owned
  RadialGrid *rad;   // not owned
  int size;
  double radii;
  double origin[3];
  std::vector<double> points;  // [size][3], radial-major: i * nang + j
  std::vector<double> weights;
  AtomicGrid(AngularGrid *a, RadialGrid *r, const double *R);
};

// Everything the Poisson pipeline needs about one atomic grid, copied out of
// the caller's RadialGrid / RTransform / AngularGrid objects so the molecular
// grid never dangles.
struct AtomLayout {
  RTParams rt;
  int nrad = 0, nang = 0, point_off = 0;
  double center[3];
  std::vector<double> r, wr, j1, j2, j3, sigma;  // per radial shell
  std::vector<double> ang;                        // [nang][3] unit vectors
};

struct PoissonPlan;  // device tables of the Poisson pipeline (capi_grid.cu)

// lmax argument meaning "per atom: lebedev_precision(nang) / 2".
constexpr int kLmaxPerAtom = -2;

// The molecular grid: concatenated atomic grids plus Becke cell weights.
struct BeckeGrid {
  int ncenter = 0;
  int size = 0;
  int ablmax = 0;
  double abldep = 1e-6;
  std::vector<double> radii, origin, points, weights, becke_weights;
  std::vector<AtomicGrid> atgrid;     // copies (share nothing with the caller)
  std::vector<int> atom_offset;       // ncenter + 1 prefix offsets
  std::vector<AtomLayout> layout;     // empty for grids read from points
  DeviceGrid dev;                     // device mirror (points SoA, weights)
  PoissonPlan *poisson = nullptr;     // cached for the last lmax used
  double poisson_tol = 0.0;           // truncation tolerance of the potential evaluation
  unsigned generation = 0;            // bumped when the centres move (napmo_grid_set_centers)
  BeckeGrid() = default;
  ~BeckeGrid();
};

// ------------------------------------------------------------------------ GTO
struct PrimitiveGaussian {
  int l[3];
  double origin[3];
  double zeta, coeff, norma;
  PrimitiveGaussian(const int *ll, const double *A, double z, double c);
};

double overlap_primitive(const PrimitiveGaussian &a, const PrimitiveGaussian &b);
// Overlap and kinetic-energy integrals of two primitives, and the normalised
// contracted matrices S, T [n][n] of a basis.
void one_body_primitive(const PrimitiveGaussian &a, const PrimitiveGaussian &b, double *S,
                        double *T);

struct ContractedGaussian {
  int l[3];
  double origin[3];
  double norma = 1.0;
  std::vector<PrimitiveGaussian> prim;
  ContractedGaussian(PrimitiveGaussian **p, int n);
  double overlap(const ContractedGaussian &o) const;
};

struct BasisSet {
  std::vector<ContractedGaussian> cont;
  int max_l = 0, max_nprim = 0;
  DeviceBasis dev;  // packed shells, uploaded lazily
  bool dev_valid = false;
  ~BasisSet();
};

void one_body_matrices(const std::vector<ContractedGaussian> &cont, double *S, double *T);

// Packs a list of contracted functions into shells for the device kernels.
void pack_basis(const std::vector<ContractedGaussian> &cont, HostBasisPack *out);

// ------------------------------------------------------------ cubic splines
struct Extrapolation;
struct CubicSpline {
  Extrapolation *ext;  // not owned
  RTransform *rtf;     // not owned
  double first_x, last_x;
  double *y, *dt;  // caller-owned arrays (the Python wrapper keeps them alive)
  int n;
  CubicSpline(double *y_, double *dt_, Extrapolation *e, RTransform *r, int n_);
  double eval(double x) const;
  double eval_deriv(double x) const;
};

struct Extrapolation {
  virtual ~Extrapolation() {}
  virtual void prepare(CubicSpline *cs) = 0;
  virtual double eval_left(double x) = 0;
  virtual double eval_right(double x) = 0;
  virtual double deriv_left(double x) = 0;
  virtual double deriv_right(double x) = 0;
  virtual bool has_tail() = 0;
};

struct ZeroExtrapolation : Extrapolation {
  void prepare(CubicSpline *) override {}
  double eval_left(double) override { return 0.0; }
  double eval_right(double) override { return 0.0; }
  double deriv_left(double) override { return 0.0; }
  double deriv_right(double) override { return 0.0; }
  bool has_tail() override { return false; }
};

struct CuspExtrapolation : Extrapolation {
  double a0 = 0, b0 = 0, x0 = 0;
  void prepare(CubicSpline *cs) override;
  double eval_left(double x) override { return a0 * exp(b0 * (x - x0)); }
  double eval_right(double) override { return 0.0; }
  double deriv_left(double x) override { return a0 * b0 * exp(b0 * (x - x0)); }
  double deriv_right(double) override { return 0.0; }
  bool has_tail() override { return false; }
};

struct PowerExtrapolation : Extrapolation {
  double power, amp = 0;
  explicit PowerExtrapolation(double p) : power(p) {}
  void prepare(CubicSpline *cs) override;
  double eval_left(double) override { return 0.0; }
  double eval_right(double x) override { return amp * pow(x, power); }
  double deriv_left(double) override { return 0.0; }
  double deriv_right(double x) override { return amp * power * pow(x, power - 1); }
  bool has_tail() override { return true; }
};

struct PotentialExtrapolation : Extrapolation {
  long l;
  double amp_left = 0, amp_right = 0;
  explicit PotentialExtrapolation(long ll) : l(ll) {}
  void prepare(CubicSpline *cs) override;
  double eval_left(double x) override { return amp_left * pow(x, l); }
  double eval_right(double x) override { return amp_right / pow(x, l + 1); }
  double deriv_left(double x) override {
    return l == 0 ? 0.0 : l * amp_left * pow(x, l - 1);
  }
  double deriv_right(double x) override {
    return -(l + 1) * amp_right / pow(x, l + 2);
  }
  bool has_tail() override { return true; }
};

void tridiag_sym_solve(double *mid, double *up, double *rhs, double *sol, int n);
void cubic_spline_dt(const double *y, double *dt, int n);

// Hermite finite-element integrals on unit segments (exact rationals).
double hermite_overlap2(long xmax, long i0, bool d0, long i1, bool d1);
double hermite_overlap3(long xmax, long i0, bool d0, long i1, bool d1, long i2,
                        bool d2);
// Flat copies of the per-segment tables: ov2[5][2][5][2], ov3[5][2][5][2][5][2]
// indexed by (piece, derivative) pairs; piece 0..3 = L0, L1, R0, R1, 4 = none.
void hermite_tables_export(double *ov2, double *ov3);
void build_ode2_matrix(const double *b, const double *a, const double *f,
                       const double *bcs, double *coeffs, double *rhs,
                       long npoint);

// Finite-difference stencils of the radial second derivative
// (RadialGrid::deriv2, src/grid/radial.cpp:51-192): first and second
// derivatives on a uniform axis, 7-point one-sided for the four points nearest
// either end and 9-point centred inside.  Weights from Fornberg's recursion
// (B. Fornberg, Math. Comp. 51, 699 (1988)), held as integers over a common
// denominator (exact); the far end uses the mirror image.
struct Deriv2Stencils {
  double edge1[4][7], edge2[4][7];  // derivative at node j (0..3) from nodes 0..6
  double mid1[9], mid2[9];          // derivative at node 4 from nodes 0..8
  double den_edge1, den_edge2, den_mid1, den_mid2;
};
const Deriv2Stencils &deriv2_stencils();

// (1/r) d^2/dr^2 (r f) = f'' + (2/r) f' on a Becke-Chebyshev radial grid
// r = radii (1 + cos w) / (1 - cos w), w_k = (k + 1) pi / (n + 1), f sampled at
// the n points r (ascending; r[n-1-k] belongs to w_k).  n >= 8.
void radial_deriv2(const double *r, int n, double radii, const double *f, double *out);

// Real solid harmonics of a 3-vector given as (z, x, y) in out[0..2]; fills
// out[3..] for l = 2..lmax (horton ordering: m = 0, then cos/sin pairs).
void pure_polynomials(double *out, long lmax);

}  // namespace napmo
