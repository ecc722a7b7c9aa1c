// Host-side construction of grids, basis sets, splines and the Hermite FEM
// matrix.  See host.h for the division of labour between host and device.
#include "host.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "common.h"
#include "solid_harmonics.h"

namespace napmo {

// ------------------------------------------------------------------ errors
static thread_local int g_last_code = 0;
static thread_local std::string g_last_msg;

int set_error(int code, const std::string &msg) {
  g_last_code = code;
  g_last_msg = msg;
  return code;
}
void clear_error() {
  g_last_code = 0;
  g_last_msg.clear();
}
int last_error(char *buf, int len) {
  if (buf && len > 0) {
    std::strncpy(buf, g_last_msg.c_str(), (size_t)len - 1);
    buf[len - 1] = '\0';
  }
  int c = g_last_code;
  return c;
}

// -------------------------------------------------------------- transforms
RTParams IdentityRT::params() const { return {kRTIdentity, npoint, 0, 0, 0}; }

LinearRT::LinearRT(double a, double b, int n) : RTransform(n), rmin(a), rmax(b) {
  if (n < 2) throw std::domain_error("A radial grid consists of at least two points.");
  if (rmin >= rmax) throw std::domain_error("rmin must be below rmax.");
  alpha = (rmax - rmin) / (npoint - 1);
}
RTParams LinearRT::params() const { return {kRTLinear, npoint, rmin, alpha, 0}; }

ExpRT::ExpRT(double a, double b, int n) : RTransform(n), rmin(a), rmax(b) {
  if (n < 2) throw std::domain_error("A radial grid consists of at least two points.");
  if (rmin >= rmax) throw std::domain_error("rmin must be below rmax.");
  if (rmin <= 0.0 || rmax <= 0.0)
    throw std::domain_error("The minimum and maximum radii must be positive.");
  alpha = log(rmax / rmin) / (npoint - 1);
}
RTParams ExpRT::params() const { return {kRTExp, npoint, rmin, alpha, 0}; }

ShiftedExpRT::ShiftedExpRT(double a, double s, double b, int n)
    : RTransform(n), rmin(a), rshift(s), rmax(b) {
  if (n < 2) throw std::domain_error("A radial grid consists of at least two points.");
  if (rmin >= rmax) throw std::domain_error("rmin must be below rmax.");
  if (rmin <= 0.0 || rmax <= 0.0)
    throw std::domain_error("The minimum and maximum radii must be positive.");
  r0 = rmin + rshift;
  if (r0 <= 0.0) throw std::domain_error("The parameter r0 must be positive.");
  alpha = log((rmax + rshift) / r0) / (npoint - 1);
}
RTParams ShiftedExpRT::params() const {
  return {kRTShiftedExp, npoint, r0, rshift, alpha};
}

PowerRT::PowerRT(double a, double b, int n) : RTransform(n), rmin(a), rmax(b) {
  if (n < 2) throw std::domain_error("A radial grid consists of at least two points.");
  if (rmin >= rmax) throw std::domain_error("rmin must be below rmax.");
  if (rmin <= 0.0 || rmax <= 0.0)
    throw std::domain_error("The minimum and maximum radii must be positive.");
  power = (log(rmax) - log(rmin)) / log(npoint);
  if (power < 2.0)
    throw std::domain_error("Power must be at least two for a decent intgration.");
}
RTParams PowerRT::params() const { return {kRTPower, npoint, rmin, power, 0}; }

RTParams ChebyshevRT::params() const { return {kRTChebyshev, npoint, radii, z, 0}; }

// ----------------------------------------------------------------- Lebedev
struct LebedevOrbit {
  int order;
  int code;
  double a, b, v;
};
#include "lebedev_orbits.inc"

// Expands one octahedral orbit.  A template places the generating values in
// (x, y, z); the sign pattern then runs over its non-zero slots, the first
// listed slot being the most significant bit and '+' preceding '-'.  Zero
// coordinates are never negated.  The template and sign orders reproduce the
// point order of the Lebedev-Laikov reference tables, which fixes nAPMO's
// point index (radial-major, then angular).
static int expand_orbit(int code, double a, double b, double v, double *x,
                        double *y, double *z, double *w) {
  struct Tmpl {
    double c[3];
    int order[3];
    int nsign;
  };
  Tmpl t[6];
  int nt = 0;
  auto add = [&](double cx, double cy, double cz, int o0, int o1, int o2, int ns) {
    t[nt].c[0] = cx;
    t[nt].c[1] = cy;
    t[nt].c[2] = cz;
    t[nt].order[0] = o0;
    t[nt].order[1] = o1;
    t[nt].order[2] = o2;
    t[nt].nsign = ns;
    nt++;
  };
  switch (code) {
    case 1:
      add(1.0, 0.0, 0.0, 0, -1, -1, 1);
      add(0.0, 1.0, 0.0, 1, -1, -1, 1);
      add(0.0, 0.0, 1.0, 2, -1, -1, 1);
      break;
    case 2: {
      const double q = 1.0 / sqrt(2.0);
      add(0.0, q, q, 1, 2, -1, 2);
      add(q, 0.0, q, 0, 2, -1, 2);
      add(q, q, 0.0, 0, 1, -1, 2);
      break;
    }
    case 3: {
      const double q = 1.0 / sqrt(3.0);
      add(q, q, q, 0, 1, 2, 3);
      break;
    }
    case 4: {
      const double c = sqrt(1.0 - 2.0 * a * a);
      add(a, a, c, 0, 1, 2, 3);
      add(a, c, a, 0, 2, 1, 3);
      add(c, a, a, 1, 2, 0, 3);
      break;
    }
    case 5: {
      const double c = sqrt(1.0 - a * a);
      add(a, c, 0.0, 0, 1, -1, 2);
      add(c, a, 0.0, 0, 1, -1, 2);
      add(a, 0.0, c, 0, 2, -1, 2);
      add(c, 0.0, a, 0, 2, -1, 2);
      add(0.0, a, c, 1, 2, -1, 2);
      add(0.0, c, a, 1, 2, -1, 2);
      break;
    }
    case 6: {
      const double c = sqrt(1.0 - a * a - b * b);
      add(a, b, c, 0, 1, 2, 3);
      add(a, c, b, 0, 1, 2, 3);
      add(b, a, c, 0, 1, 2, 3);
      add(b, c, a, 0, 1, 2, 3);
      add(c, a, b, 0, 1, 2, 3);
      add(c, b, a, 0, 1, 2, 3);
      break;
    }
    default:
      return -1;
  }
  int n = 0;
  for (int it = 0; it < nt; ++it) {
    const int ns = t[it].nsign;
    for (int mask = 0; mask < (1 << ns); ++mask) {
      double p[3] = {t[it].c[0], t[it].c[1], t[it].c[2]};
      for (int s = 0; s < ns; ++s) {
        if (mask & (1 << (ns - 1 - s))) p[t[it].order[s]] = -p[t[it].order[s]];
      }
      x[n] = p[0];
      y[n] = p[1];
      z[n] = p[2];
      w[n] = v;
      n++;
    }
  }
  return n;
}

bool lebedev_rule(int order, double *x, double *y, double *z, double *w) {
  int n = 0;
  bool found = false;
  for (const LebedevOrbit &o : kLebedevOrbits) {
    if (o.order != order) continue;
    found = true;
    n += expand_orbit(o.code, o.a, o.b, o.v, x + n, y + n, z + n, w + n);
  }
  return found && n == order;
}

int lebedev_precision(int order) {
  static const int table[][2] = {
      {6, 3},     {14, 5},    {26, 7},    {38, 9},    {50, 11},   {74, 13},
      {86, 15},   {110, 17},  {146, 19},  {170, 21},  {194, 23},  {230, 25},
      {266, 27},  {302, 29},  {350, 31},  {434, 35},  {590, 41},  {770, 47},
      {974, 53},  {1202, 59}, {1454, 65}, {1730, 71}, {2030, 77}, {2354, 83},
      {2702, 89}, {3074, 95}, {3470, 101}, {3890, 107}, {4334, 113},
      {4802, 119}, {5294, 125}, {5810, 131}};
  for (auto &e : table)
    if (e[0] == order) return e[1];
  return -1;
}

// ------------------------------------------------------------------- grids
RadialGrid::RadialGrid(RTransform *rt, double rad) : rtf(rt), radii(rad) {
  const int n = rt->npoint;
  points.resize(n);
  weights.resize(n);
  const double PI_4 = M_PI * 4.0;
  for (int i = 0; i < n; ++i) {
    double t = i;
    points[i] = rt->radius(t);
    weights[i] = PI_4 * rt->deriv(t) * points[i] * points[i];
  }
}

double RadialGrid::integrate(int segments, const double *f) const {
  const int n = (int)points.size();
  double out = 0.0;
  for (int i = 0; i < n; ++i) {
    double v = f[i];
    for (int s = 1; s < segments; ++s) v *= f[s * n + i];
    out += v * weights[i];
  }
  return out;
}

AngularGrid::AngularGrid(int order) : lorder(order) {
  points.assign((size_t)order * 3, 0.0);
  weights.assign(order, 0.0);
  std::vector<double> x(order), y(order), z(order);
  if (!lebedev_rule(order, x.data(), y.data(), z.data(), weights.data()))
    throw std::domain_error("Unknown Lebedev order " + std::to_string(order));
  for (int i = 0; i < order; ++i) {
    points[i * 3 + 0] = x[i];
    points[i * 3 + 1] = y[i];
    points[i * 3 + 2] = z[i];
  }
}

AtomicGrid::AtomicGrid(AngularGrid *a, RadialGrid *r, const double *R)
    : ang(a), rad(r) {
  const int nrad = (int)r->points.size();
  const int nang = a->lorder;
  size = nrad * nang;
  radii = r->radii;
  origin[0] = R[0];
  origin[1] = R[1];
  origin[2] = R[2];
  points.resize((size_t)size * 3);
  weights.resize(size);
  for (int i = 0; i < nrad; ++i) {
    const double rp = r->points[i];
    const double rw = r->weights[i];
    for (int j = 0; j < nang; ++j) {
      const size_t k = (size_t)i * nang + j;
      points[k * 3 + 0] = a->points[j * 3 + 0] * rp + origin[0];
      points[k * 3 + 1] = a->points[j * 3 + 1] * rp + origin[1];
      points[k * 3 + 2] = a->points[j * 3 + 2] * rp + origin[2];
      weights[k] = a->weights[j] * rw;
    }
  }
}

// --------------------------------------------------------------------- GTO
static int double_factorial(int n) {
  if (n < 1) return 0;
  int out = 1;
  for (int i = n; i > 0; i -= 2) out *= i;
  return out;
}

PrimitiveGaussian::PrimitiveGaussian(const int *ll, const double *A, double z,
                                     double c)
    : zeta(z), coeff(c), norma(1.0) {
  int L = 0;
  for (int i = 0; i < 3; ++i) {
    l[i] = ll[i];
    origin[i] = A[i];
    L += l[i];
  }
  // N = (2 zeta / pi)^(3/4) / sqrt(prod (2 l_i - 1)!! / (4 zeta)^L)
  const int dfac = double_factorial(abs(2 * l[0] - 1)) *
                   double_factorial(abs(2 * l[1] - 1)) *
                   double_factorial(abs(2 * l[2] - 1));
  norma = pow(2.0 * zeta / M_PI, 0.75) / sqrt(dfac / pow(4.0 * zeta, L));
}

// Obara-Saika overlap of two Cartesian primitives: the 1D Hermite overlap
// tables E_ij obey E_{i+1,j} = X_PA E_ij + (i E_{i-1,j} + j E_{i,j-1}) / 2p and
// the same recursion with X_PB on the second index; the 3D overlap is the
// product of the three 1D factors times exp(-mu R_AB^2) (pi/p)^{3/2}.
double overlap_primitive(const PrimitiveGaussian &a, const PrimitiveGaussian &b) {
  const double p = a.zeta + b.zeta;
  const double pinv = 1.0 / p;
  double AB2 = 0.0;
  double S1[3];
  for (int d = 0; d < 3; ++d) {
    const double AB = a.origin[d] - b.origin[d];
    const double P = (a.zeta * a.origin[d] + b.zeta * b.origin[d]) * pinv;
    const double PA = P - a.origin[d];
    const double PB = P - b.origin[d];
    AB2 += AB * AB;
    const int la = a.l[d], lb = b.l[d];
    double E[16][16];
    const double h = 0.5 * pinv;
    E[0][0] = 1.0;
    for (int j = 0; j < lb; ++j)
      E[0][j + 1] = PB * E[0][j] + (j > 0 ? j * h * E[0][j - 1] : 0.0);
    for (int i = 0; i < la; ++i) {
      for (int j = 0; j <= lb; ++j) {
        double v = PA * E[i][j];
        if (i > 0) v += i * h * E[i - 1][j];
        if (j > 0) v += j * h * E[i][j - 1];
        E[i + 1][j] = v;
      }
    }
    S1[d] = E[la][lb];
  }
  const double pre = exp(-a.zeta * b.zeta * AB2 * pinv) *
                     (sqrt(M_PI * pinv) * M_PI * pinv * a.coeff * b.coeff *
                      a.norma * b.norma);
  return pre * S1[0] * S1[1] * S1[2];
}

// Overlap and kinetic energy of two Cartesian primitives (coefficients and
// primitive norms included).  The 1D Obara-Saika overlaps E[i][j] are built up
// to la + 1, lb + 1; per axis the kinetic term is
//   t(i, j) = 1/2 <d/dx a|d/dx b> = 1/2 [ i j E(i-1, j-1) - 2 zb i E(i-1, j+1)
//                                       - 2 za j E(i+1, j-1) + 4 za zb E(i+1, j+1) ]
// and T = tx Sy Sz + Sx ty Sz + Sx Sy tz.
void one_body_primitive(const PrimitiveGaussian &a, const PrimitiveGaussian &b, double *S,
                        double *T) {
  const double p = a.zeta + b.zeta;
  const double pinv = 1.0 / p;
  double AB2 = 0.0, S1[3], T1[3];
  for (int d = 0; d < 3; ++d) {
    const double AB = a.origin[d] - b.origin[d];
    const double P = (a.zeta * a.origin[d] + b.zeta * b.origin[d]) * pinv;
    const double PA = P - a.origin[d], PB = P - b.origin[d];
    AB2 += AB * AB;
    const int la = a.l[d] + 1, lb = b.l[d] + 1;
    double E[17][17];
    const double h = 0.5 * pinv;
    E[0][0] = 1.0;
    for (int j = 0; j < lb; ++j)
      E[0][j + 1] = PB * E[0][j] + (j > 0 ? j * h * E[0][j - 1] : 0.0);
    for (int i = 0; i < la; ++i)
      for (int j = 0; j <= lb; ++j) {
        double v = PA * E[i][j];
        if (i > 0) v += i * h * E[i - 1][j];
        if (j > 0) v += j * h * E[i][j - 1];
        E[i + 1][j] = v;
      }
    const int i = a.l[d], j = b.l[d];
    S1[d] = E[i][j];
    double t = 4.0 * a.zeta * b.zeta * E[i + 1][j + 1];
    if (i > 0 && j > 0) t += i * j * E[i - 1][j - 1];
    if (i > 0) t -= 2.0 * b.zeta * i * E[i - 1][j + 1];
    if (j > 0) t -= 2.0 * a.zeta * j * E[i + 1][j - 1];
    T1[d] = 0.5 * t;
  }
  const double pre = exp(-a.zeta * b.zeta * AB2 * pinv) *
                     (sqrt(M_PI * pinv) * M_PI * pinv * a.coeff * b.coeff * a.norma * b.norma);
  *S = pre * S1[0] * S1[1] * S1[2];
  *T = pre * (T1[0] * S1[1] * S1[2] + S1[0] * T1[1] * S1[2] + S1[0] * S1[1] * T1[2]);
}

void one_body_matrices(const std::vector<ContractedGaussian> &cont, double *S, double *T) {
  const size_t n = cont.size();
  for (size_t m = 0; m < n; ++m)
    for (size_t k = 0; k <= m; ++k) {
      double s = 0.0, t = 0.0;
      for (const auto &pa : cont[m].prim)
        for (const auto &pb : cont[k].prim) {
          double ps, pt;
          one_body_primitive(pa, pb, &ps, &pt);
          s += ps;
          t += pt;
        }
      const double nn = cont[m].norma * cont[k].norma;
      S[m * n + k] = S[k * n + m] = s * nn;
      T[m * n + k] = T[k * n + m] = t * nn;
    }
}

ContractedGaussian::ContractedGaussian(PrimitiveGaussian **p, int n) {
  for (int i = 0; i < 3; ++i) {
    origin[i] = p[0]->origin[i];
    l[i] = p[0]->l[i];
  }
  for (int i = 0; i < n; ++i) prim.push_back(*p[i]);
  norma = 1.0 / sqrt(overlap(*this));
}

double ContractedGaussian::overlap(const ContractedGaussian &o) const {
  double out = 0.0;
  for (const auto &pa : prim)
    for (const auto &pb : o.prim) out += overlap_primitive(pa, pb);
  return out * norma * o.norma;
}

void pack_basis(const std::vector<ContractedGaussian> &cont, HostBasisPack *out) {
  HostBasisPack &pk = *out;
  pk = HostBasisPack();
  pk.nfunc = (int)cont.size();
  size_t f = 0;
  while (f < cont.size()) {
    const ContractedGaussian &c0 = cont[f];
    const int L = c0.l[0] + c0.l[1] + c0.l[2];
    const int np = (int)c0.prim.size();
    const int maxcomp = (L + 1) * (L + 2) / 2;
    size_t g = f + 1;
    while (g < cont.size() && (int)(g - f) < maxcomp) {
      const ContractedGaussian &c = cont[g];
      if (c.l[0] + c.l[1] + c.l[2] != L || (int)c.prim.size() != np) break;
      bool same = c.origin[0] == c0.origin[0] && c.origin[1] == c0.origin[1] &&
                  c.origin[2] == c0.origin[2];
      for (int k = 0; same && k < np; ++k) same = c.prim[k].zeta == c0.prim[k].zeta;
      if (!same) break;
      ++g;
    }
    const int ncomp = (int)(g - f);
    pk.shell_info.push_back((int)f);
    pk.shell_info.push_back(ncomp);
    pk.shell_info.push_back((int)pk.prim_zeta.size());
    pk.shell_info.push_back(np);
    pk.shell_info.push_back((int)pk.coef.size());
    pk.shell_info.push_back(L);
    double zmin = c0.prim[0].zeta;
    for (int k = 1; k < np; ++k) zmin = std::min(zmin, c0.prim[k].zeta);
    for (int d = 0; d < 3; ++d) pk.shell_center.push_back(c0.origin[d]);
    pk.shell_center.push_back(zmin);
    for (int k = 0; k < np; ++k) pk.prim_zeta.push_back(c0.prim[k].zeta);
    for (size_t h = f; h < g; ++h) {
      const ContractedGaussian &c = cont[h];
      for (int k = 0; k < np; ++k)
        pk.coef.push_back(c.prim[k].coeff * c.prim[k].norma * c.norma);
    }
    pk.max_nprim = std::max(pk.max_nprim, np);
    pk.max_l = std::max(pk.max_l, L);
    pk.nshell++;
    f = g;
  }
  for (const auto &c : cont)
    for (int d = 0; d < 3; ++d) pk.func_l.push_back(c.l[d]);
}

// ------------------------------------------------------------ cubic spline
CubicSpline::CubicSpline(double *y_, double *dt_, Extrapolation *e, RTransform *r,
                         int n_)
    : ext(e), rtf(r), first_x(0.0), last_x(0.0), y(y_), dt(dt_), n(n_) {
  first_x = rtf->radius(0);
  last_x = rtf->radius(n - 1);
  ext->prepare(this);
}

double CubicSpline::eval(double x) const {
  if (x < first_x) return ext->eval_left(x);
  if (x > last_x) return ext->eval_right(x);
  const double t = rtf->inv(x);
  int j = static_cast<int>(floor(t));
  if (j == n - 1) j = n - 2;
  if (j < 0) j = 0;
  const double u = t - j;
  const double z = y[j + 1] - y[j];
  return y[j] + u * (dt[j] + u * (3 * z - 2 * dt[j] - dt[j + 1] +
                                  u * (-2 * z + dt[j] + dt[j + 1])));
}

double CubicSpline::eval_deriv(double x) const {
  if (x < first_x) return ext->deriv_left(x);
  if (x > last_x) return ext->deriv_right(x);
  const double t = rtf->inv(x);
  int j = (int)floor(t);
  if (j == n - 1) j = n - 2;
  if (j < 0) j = 0;
  const double u = t - j;
  const double z = y[j + 1] - y[j];
  double d = dt[j] + u * (6 * z - 4 * dt[j] - 2 * dt[j + 1] +
                          u * (-6 * z + 3 * dt[j] + 3 * dt[j + 1]));
  return d / rtf->deriv(t);
}

void CuspExtrapolation::prepare(CubicSpline *cs) {
  x0 = cs->first_x;
  if (fabs(cs->y[0]) < 0.00001) {
    a0 = 0;
    b0 = 0;
  } else {
    a0 = cs->y[0];
    b0 = cs->dt[0] / cs->y[0] / cs->rtf->deriv(0);
  }
}

void PowerExtrapolation::prepare(CubicSpline *cs) {
  amp = cs->y[cs->n - 1] * pow(cs->last_x, -power);
}

void PotentialExtrapolation::prepare(CubicSpline *cs) {
  amp_left = cs->y[0] / pow(cs->first_x, l);
  amp_right = cs->y[cs->n - 1] * pow(cs->last_x, l + 1);
}

// Symmetric tridiagonal solve by forward elimination / back substitution
// (Thomas algorithm); `up` and `rhs` are overwritten.
void tridiag_sym_solve(double *mid, double *up, double *rhs, double *sol, int n) {
  double prev_up = up[0];
  double next_up = 0.0;
  up[0] /= mid[0];
  rhs[0] /= mid[0];
  for (int i = 1; i < n; i++) {
    const double den = mid[i] - up[i - 1] * prev_up;
    if (i < n - 1) {
      next_up = up[i];
      up[i] /= den;
    }
    rhs[i] = (rhs[i] - rhs[i - 1] * prev_up) / den;
    prev_up = next_up;
  }
  sol[n - 1] = rhs[n - 1];
  for (int i = n - 2; i >= 0; i--) sol[i] = rhs[i] - up[i] * sol[i + 1];
}

// Derivatives (on the uniform t-axis) of the cubic spline through y with
// continuous second derivative and natural-like end rows (2, 1 / 1, 2).
void cubic_spline_dt(const double *y, double *dt, int n) {
  std::vector<double> mid(n), up(n), rhs(n);
  mid[0] = 2.0;
  up[0] = 1.0;
  rhs[0] = 3.0 * (y[1] - y[0]);
  for (int i = 1; i < n - 1; i++) {
    mid[i] = 4.0;
    up[i] = 1.0;
    rhs[i] = 3.0 * (y[i + 1] - y[i - 1]);
  }
  mid[n - 1] = 2.0;
  rhs[n - 1] = 3.0 * (y[n - 1] - y[n - 2]);
  tridiag_sym_solve(mid.data(), up.data(), rhs.data(), dt, n);
}

// ------------------------------------------------ radial second derivative
// Fornberg's recursion: c[j * (m + 1) + k] = weight of node x[j] in the k-th
// derivative at z (k <= m), nodes x[0..np-1].
static void fornberg_weights(double z, const double *x, int np, int m, double *c) {
  for (int e = 0; e < np * (m + 1); ++e) c[e] = 0.0;
  double c1 = 1.0, c4 = x[0] - z;
  c[0] = 1.0;
  for (int i = 1; i < np; ++i) {
    const int mn = i < m ? i : m;
    double c2 = 1.0;
    const double c5 = c4;
    c4 = x[i] - z;
    for (int j = 0; j < i; ++j) {
      const double c3 = x[i] - x[j];
      c2 *= c3;
      if (j == i - 1) {
        for (int k = mn; k >= 1; --k)
          c[i * (m + 1) + k] =
              c1 * (k * c[(i - 1) * (m + 1) + k - 1] - c5 * c[(i - 1) * (m + 1) + k]) / c2;
        c[i * (m + 1)] = -c1 * c5 * c[(i - 1) * (m + 1)] / c2;
      }
      for (int k = mn; k >= 1; --k)
        c[j * (m + 1) + k] = (c4 * c[j * (m + 1) + k] - k * c[j * (m + 1) + k - 1]) / c3;
      c[j * (m + 1)] = c4 * c[j * (m + 1)] / c3;
    }
    c1 = c2;
  }
}

const Deriv2Stencils &deriv2_stencils() {
  static const Deriv2Stencils st = [] {
    // common denominators of the weights: 7-point stencils are multiples of
    // 1/720 (first derivative) and 1/360 (second), 9-point ones of 1/40320
    // and 1/20160; scaled weights are exact integers
    Deriv2Stencils s;
    s.den_edge1 = 720.0;
    s.den_edge2 = 360.0;
    s.den_mid1 = 40320.0;
    s.den_mid2 = 20160.0;
    double x[9], c[9 * 3];
    for (int k = 0; k < 9; ++k) x[k] = k;
    for (int j = 0; j < 4; ++j) {
      fornberg_weights((double)j, x, 7, 2, c);
      for (int k = 0; k < 7; ++k) {
        s.edge1[j][k] = std::nearbyint(c[k * 3 + 1] * s.den_edge1);
        s.edge2[j][k] = std::nearbyint(c[k * 3 + 2] * s.den_edge2);
      }
    }
    fornberg_weights(4.0, x, 9, 2, c);
    for (int k = 0; k < 9; ++k) {
      s.mid1[k] = std::nearbyint(c[k * 3 + 1] * s.den_mid1);
      s.mid2[k] = std::nearbyint(c[k * 3 + 2] * s.den_mid2);
    }
    return s;
  }();
  return st;
}

void radial_deriv2(const double *r, int n, double radii, const double *f, double *out) {
  if (n < 8) throw std::invalid_argument("radial second derivative needs >= 8 points");
  const Deriv2Stencils &st = deriv2_stencils();
  const double H = M_PI / (n + 1.0);
  // g_k = f(w_k) = f[n - 1 - k]
  auto g = [&](int k) { return f[n - 1 - k]; };
  for (int i = 0; i < n; ++i) {
    double d1 = 0.0, d2 = 0.0;
    if (i < 4) {
      for (int k = 0; k < 7; ++k) {
        d1 += st.edge1[i][k] * g(k);
        d2 += st.edge2[i][k] * g(k);
      }
      d1 /= st.den_edge1 * H;
      d2 /= st.den_edge2 * H * H;
    } else if (i >= n - 4) {
      const int j = n - 1 - i;  // mirror of node j: first-derivative weights change sign
      for (int k = 6; k >= 0; --k) {
        d1 -= st.edge1[j][k] * g(n - 1 - k);
        d2 += st.edge2[j][k] * g(n - 1 - k);
      }
      d1 /= st.den_edge1 * H;
      d2 /= st.den_edge2 * H * H;
    } else {
      for (int k = 0; k < 9; ++k) {
        d1 += st.mid1[k] * g(i - 4 + k);
        d2 += st.mid2[k] * g(i - 4 + k);
      }
      d1 /= st.den_mid1 * H;
      d2 /= st.den_mid2 * H * H;
    }
    // dw/dr and d2w/dr2 of r(w) = radii (1 + cos w) / (1 - cos w)
    const double w = (i + 1) * H, X = cos(w), Y = sin(w), q = 1.0 - X;
    const double wr = -q * q / (2.0 * radii * Y);
    const double wrr = q * q * q * (2.0 * Y * Y - q * X) / (4.0 * radii * radii * Y * Y * Y);
    const int idx = n - 1 - i;
    out[idx] = wr * wr * d2 + (wrr + 2.0 * wr / r[idx]) * d1;
  }
}

// ----------------------------------------------------- Hermite FEM integrals
// Cubic Hermite basis on the unit segment s in [0, 1]:
//   L0 = 1 - 3s^2 + 2s^3 (value at left node), L1 = s - 2s^2 + s^3,
//   R0 = 3s^2 - 2s^3 (value at right node),     R1 = -s^2 + s^3.
// The global basis function (node c, kind k) equals Lk on [c, c+1] and Rk on
// [c-1, c].  Integrals are computed exactly as integers over 2520 = lcm(1..10)
// and converted once, so each table entry is the correctly rounded double of
// the exact rational.
namespace {
struct HermiteTables {
  // ov2[p0][d0][p1][d1], ov3[p0][d0][p1][d1][p2][d2]; polynomial id 4 = 0.
  double ov2[5][2][5][2];
  double ov3[5][2][5][2][5][2];
  HermiteTables() {
    static const long poly[5][4] = {
        {1, 0, -3, 2}, {0, 1, -2, 1}, {0, 0, 3, -2}, {0, 0, -1, 1}, {0, 0, 0, 0}};
    auto der = [](const long *c, int d, long *o) {
      for (int k = 0; k < 4; ++k) o[k] = c[k];
      if (d) {
        o[0] = c[1];
        o[1] = 2 * c[2];
        o[2] = 3 * c[3];
        o[3] = 0;
      }
    };
    auto integrate = [](const long *c, int deg) {
      long num = 0;
      for (int k = 0; k <= deg; ++k) num += c[k] * (2520 / (k + 1));
      return (double)num / 2520.0;
    };
    for (int p0 = 0; p0 < 5; ++p0)
      for (int d0 = 0; d0 < 2; ++d0)
        for (int p1 = 0; p1 < 5; ++p1)
          for (int d1 = 0; d1 < 2; ++d1) {
            long a[4], b[4], prod[7] = {0};
            der(poly[p0], d0, a);
            der(poly[p1], d1, b);
            for (int i = 0; i < 4; ++i)
              for (int j = 0; j < 4; ++j) prod[i + j] += a[i] * b[j];
            ov2[p0][d0][p1][d1] = integrate(prod, 6);
            for (int p2 = 0; p2 < 5; ++p2)
              for (int d2 = 0; d2 < 2; ++d2) {
                long c[4], prod3[10] = {0};
                der(poly[p2], d2, c);
                for (int i = 0; i < 7; ++i)
                  for (int k = 0; k < 4; ++k) prod3[i + k] += prod[i] * c[k];
                ov3[p0][d0][p1][d1][p2][d2] = integrate(prod3, 9);
              }
          }
  }
};
const HermiteTables &tables() {
  static const HermiteTables t;
  return t;
}
// Polynomial id of basis function (node c, kind k) on segment [g, g+1].
inline int piece(long c, long k, long g) {
  if (c == g) return (int)k;
  if (c == g + 1) return (int)(2 + k);
  return 4;
}
}  // namespace

void hermite_tables_export(double *ov2, double *ov3) {
  const HermiteTables &T = tables();
  std::memcpy(ov2, &T.ov2[0][0][0][0], sizeof(T.ov2));
  std::memcpy(ov3, &T.ov3[0][0][0][0][0][0], sizeof(T.ov3));
}

double hermite_overlap2(long xmax, long i0, bool d0, long i1, bool d1) {
  const long c0 = i0 / 2, k0 = i0 % 2, c1 = i1 / 2, k1 = i1 % 2;
  if (std::labs(c1 - c0) >= 2) return 0.0;
  const HermiteTables &T = tables();
  double r = 0.0;
  if (c0 >= 1 && c0 <= xmax)
    r += T.ov2[piece(c0, k0, c0 - 1)][d0][piece(c1, k1, c0 - 1)][d1];
  if (c0 >= 0 && c0 <= xmax - 1)
    r += T.ov2[piece(c0, k0, c0)][d0][piece(c1, k1, c0)][d1];
  return r;
}

double hermite_overlap3(long xmax, long i0, bool d0, long i1, bool d1, long i2,
                        bool d2) {
  const long c0 = i0 / 2, k0 = i0 % 2, c1 = i1 / 2, k1 = i1 % 2, c2 = i2 / 2,
             k2 = i2 % 2;
  if (std::labs(c1 - c0) >= 2 || std::labs(c2 - c0) >= 2) return 0.0;
  const HermiteTables &T = tables();
  double r = 0.0;
  if (c0 >= 1 && c0 <= xmax) {
    const long g = c0 - 1;
    r += T.ov3[piece(c0, k0, g)][d0][piece(c1, k1, g)][d1][piece(c2, k2, g)][d2];
  }
  if (c0 >= 0 && c0 <= xmax - 1) {
    const long g = c0;
    r += T.ov3[piece(c0, k0, g)][d0][piece(c1, k1, g)][d1][piece(c2, k2, g)][d2];
  }
  return r;
}

static inline double node_value(long x, long c, long k, bool d) {
  return (k == (long)d) ? (double)(x == c) : 0.0;
}

// Galerkin matrix of u'' + b u' + a u = f in the cubic Hermite basis on the
// t-axis (unknowns interleaved value/derivative per node), with Dirichlet or
// Neumann rows where bcs[] is not NaN (nAPMO src/horton/ode2.cpp:232-321).
void build_ode2_matrix(const double *b, const double *a, const double *f,
                       const double *bcs, double *coeffs, double *rhs,
                       long npoint) {
  const long nfn = 2 * npoint;
  long skip[2] = {-1, -1};
  int nskip = 0;
  auto note_skip = [&](long row) {
    if (nskip < 2) skip[nskip] = row;
    nskip++;
  };
  if (bcs[0] == bcs[0]) {
    coeffs[0] = 1;
    rhs[0] = bcs[0];
    note_skip(0);
  }
  if (bcs[1] == bcs[1]) {
    coeffs[nfn + 1] = 1;
    rhs[1] = bcs[1];
    note_skip(1);
  }
  if (bcs[2] == bcs[2]) {
    coeffs[nfn * (nfn - 1) - 2] = 1;
    rhs[nfn - 2] = bcs[2];
    note_skip(nfn - 2);
  }
  if (bcs[3] == bcs[3]) {
    coeffs[nfn * nfn - 1] = 1;
    rhs[nfn - 1] = bcs[3];
    note_skip(nfn - 1);
  }
  const long xmax = npoint - 1;
  for (long row = 0; row < nfn; row++) {
    if (row == skip[0] || row == skip[1]) continue;
    long lo = 2 * (row / 2 - 1);
    if (lo < 0) lo = 0;
    long hi = 2 * (row / 2 + 2);
    if (hi > nfn) hi = nfn;
    for (long col = lo; col < hi; col++) {
      double *c = coeffs + (row * nfn + col);
      *c -= hermite_overlap2(xmax, row, true, col, true);
      for (long k = lo; k < hi; k++) {
        if (b[k] != 0) *c += b[k] * hermite_overlap3(xmax, row, false, col, true, k, false);
        if (a[k] != 0) *c += a[k] * hermite_overlap3(xmax, row, false, col, false, k, false);
      }
      *c += node_value(xmax, row / 2, row % 2, false) *
            node_value(xmax, col / 2, col % 2, true);
      *c -= node_value(0, row / 2, row % 2, false) *
            node_value(0, col / 2, col % 2, true);
    }
    double *r = rhs + row;
    for (long k = lo; k < hi; k++) {
      if (f[k] != 0) *r += f[k] * hermite_overlap2(xmax, row, false, k, false);
    }
  }
}

void pure_polynomials(double *out, long lmax) { solid_harmonics(out, lmax); }

}  // namespace napmo
