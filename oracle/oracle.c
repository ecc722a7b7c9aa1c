/*
 * ORACLE -- test infrastructure only.  A plain-C, single-file restatement of
 * nAPMO's CPU algorithm for the grid-quadrature path, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU baseline as the checker.
 * Nothing in the napmo_b200 package links, loads or calls it.
 *
 * Every function follows the reference operation order (compiled like nAPMO:
 * -O2 without -march, so no FMA contraction) and cites the file:line it
 * restates (paths relative to the nAPMO source tree).  Pinning: the radial
 * transforms, Lebedev rules, GTO values/norms, spline and ODE builders are
 * compared against nAPMO's own compiled sources (oracle/_ref) where those
 * build here; the Becke weights and quadratures (Eigen-bound in nAPMO, not
 * buildable here) are pinned by nAPMO's known-answer tests (single-centre
 * Coulomb integral 0.77461, spherical averages, radial integrals) and by
 * the bit-exact agreement of this restatement with the GPU kernels.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------ transforms */
/* src/horton/rtransform.cpp:308-341 (Chebyshev), :257-299 (Power) */
double orc_cheb_radius(double radii, int n, double t) {
  double z = M_PI / (n + 1);
  t = n - t;
  double aux = cos(t * z);
  return radii * (1 + aux) / (1 - aux);
}
double orc_cheb_deriv(double radii, int n, double t) {
  double z = M_PI / (n + 1);
  t = n - t;
  double aux = t * z;
  return (2 * radii * z * sin(aux)) / pow(cos(aux) - 1, 2);
}
double orc_cheb_deriv2(double radii, int n, double t) {
  double z = M_PI / (n + 1);
  t = n - t;
  double aux = t * z;
  return 0.5 * z * z * radii * (2 + cos(aux)) * pow(1 / sin(aux * 0.5), 4);
}
double orc_cheb_deriv3(double radii, int n, double t) {
  double z = M_PI / (n + 1);
  t = n - t;
  double aux = t * z;
  double aux_2 = aux * 0.5;
  return 0.25 * z * z * z * radii * (11 * cos(aux_2) + cos(1.5 * aux)) *
         pow(1 / sin(aux_2), 5);
}
double orc_cheb_inv(double radii, int n, double r) {
  double z = M_PI / (n + 1);
  return -(acos((r - radii) / (r + radii)) / z) + n;
}
double orc_power_param(double rmin, double rmax, int n) {
  return (log(rmax) - log(rmin)) / log(n);
}
double orc_power_radius(double rmin, double power, double t) { return rmin * pow(t + 1, power); }
double orc_power_deriv(double rmin, double power, double t) {
  return power * rmin * pow(t + 1, power - 1);
}

/* src/grid/radial.cpp:14-29: r_i = radius(i), w_i = 4 pi deriv(i) r_i^2.
 * kind 0 = Chebyshev(p0 = radii), 1 = Power(p0 = rmin, p1 = rmax). */
void orc_radial_grid(int kind, double p0, double p1, int n, double *r, double *w) {
  double PI_4 = M_PI * 4.0;
  double power = kind == 1 ? orc_power_param(p0, p1, n) : 0.0;
  for (int i = 0; i < n; ++i) {
    double x = i;
    double d;
    if (kind == 0) {
      r[i] = orc_cheb_radius(p0, n, x);
      d = orc_cheb_deriv(p0, n, x);
    } else {
      r[i] = orc_power_radius(p0, power, x);
      d = orc_power_deriv(p0, power, x);
    }
    w[i] = PI_4 * d * r[i] * r[i];
  }
}

/* ------------------------------------------------------------- Lebedev */
/* Orbit expansion of the Lebedev-Laikov rules in the order of the published
 * tables (src/grid/sphere_lebedev_rule.cpp: gen_oh), written out per code. */
typedef struct {
  int order;
  int code;
  double a, b, v;
} LebedevOrbit;
#include "../napmo_b200/csrc/lebedev_orbits.inc"

static int put(double *x, double *y, double *z, double *w, int n, double px, double py,
               double pz, double v) {
  x[n] = px; y[n] = py; z[n] = pz; w[n] = v;
  return n + 1;
}

static int orbit(int code, double a, double b, double v, double *x, double *y, double *z,
                 double *w) {
  int n = 0;
  double c;
  switch (code) {
    case 1:
      a = 1.0;
      n = put(x, y, z, w, n, a, 0.0, 0.0, v);  n = put(x, y, z, w, n, -a, 0.0, 0.0, v);
      n = put(x, y, z, w, n, 0.0, a, 0.0, v);  n = put(x, y, z, w, n, 0.0, -a, 0.0, v);
      n = put(x, y, z, w, n, 0.0, 0.0, a, v);  n = put(x, y, z, w, n, 0.0, 0.0, -a, v);
      break;
    case 2:
      a = 1.0 / sqrt(2.0);
      n = put(x, y, z, w, n, 0.0, a, a, v);   n = put(x, y, z, w, n, 0.0, a, -a, v);
      n = put(x, y, z, w, n, 0.0, -a, a, v);  n = put(x, y, z, w, n, 0.0, -a, -a, v);
      n = put(x, y, z, w, n, a, 0.0, a, v);   n = put(x, y, z, w, n, a, 0.0, -a, v);
      n = put(x, y, z, w, n, -a, 0.0, a, v);  n = put(x, y, z, w, n, -a, 0.0, -a, v);
      n = put(x, y, z, w, n, a, a, 0.0, v);   n = put(x, y, z, w, n, a, -a, 0.0, v);
      n = put(x, y, z, w, n, -a, a, 0.0, v);  n = put(x, y, z, w, n, -a, -a, 0.0, v);
      break;
    case 3:
      a = 1.0 / sqrt(3.0);
      for (int s = 0; s < 8; ++s)
        n = put(x, y, z, w, n, (s & 4) ? -a : a, (s & 2) ? -a : a, (s & 1) ? -a : a, v);
      break;
    case 4:
      b = sqrt(1.0 - 2.0 * a * a);
      for (int s = 0; s < 8; ++s)  /* (a, a, b): x, y, z */
        n = put(x, y, z, w, n, (s & 4) ? -a : a, (s & 2) ? -a : a, (s & 1) ? -b : b, v);
      for (int s = 0; s < 8; ++s)  /* (a, b, a): x, z, y */
        n = put(x, y, z, w, n, (s & 4) ? -a : a, (s & 1) ? -b : b, (s & 2) ? -a : a, v);
      for (int s = 0; s < 8; ++s)  /* (b, a, a): y, z, x */
        n = put(x, y, z, w, n, (s & 1) ? -b : b, (s & 4) ? -a : a, (s & 2) ? -a : a, v);
      break;
    case 5:
      b = sqrt(1.0 - a * a);
      {
        double t[6][3] = {{a, b, 0}, {b, a, 0}, {a, 0, b}, {b, 0, a}, {0, a, b}, {0, b, a}};
        for (int k = 0; k < 6; ++k) {
          for (int s = 0; s < 4; ++s) {
            double p[3] = {t[k][0], t[k][1], t[k][2]};
            int first = -1, second = -1;
            for (int d = 0; d < 3; ++d)
              if (p[d] != 0.0) { if (first < 0) first = d; else second = d; }
            if (s & 2) p[first] = -p[first];
            if (s & 1) p[second] = -p[second];
            n = put(x, y, z, w, n, p[0], p[1], p[2], v);
          }
        }
      }
      break;
    case 6:
      c = sqrt(1.0 - a * a - b * b);
      {
        double t[6][3] = {{a, b, c}, {a, c, b}, {b, a, c}, {b, c, a}, {c, a, b}, {c, b, a}};
        for (int k = 0; k < 6; ++k)
          for (int s = 0; s < 8; ++s)
            n = put(x, y, z, w, n, (s & 4) ? -t[k][0] : t[k][0], (s & 2) ? -t[k][1] : t[k][1],
                    (s & 1) ? -t[k][2] : t[k][2], v);
      }
      break;
  }
  return n;
}

int orc_lebedev(int order, double *x, double *y, double *z, double *w) {
  int n = 0;
  for (size_t i = 0; i < sizeof(kLebedevOrbits) / sizeof(kLebedevOrbits[0]); ++i) {
    const LebedevOrbit *o = &kLebedevOrbits[i];
    if (o->order == order) n += orbit(o->code, o->a, o->b, o->v, x + n, y + n, z + n, w + n);
  }
  return n;
}

/* src/grid/atomic_grid.cpp:12-51: radial-major points u_j r_i + R. */
void orc_atomic_grid(int nrad, const double *r, const double *wr, int nang, const double *ax,
                     const double *ay, const double *az, const double *aw, const double *R,
                     double *points, double *weights) {
  for (int i = 0; i < nrad; ++i) {
    double rp = r[i], rw = wr[i];
    for (int j = 0; j < nang; ++j) {
      unsigned int aux = i * nang + j, idy = aux * 3;
      points[idy + 0] = ax[j] * rp + R[0];
      points[idy + 1] = ay[j] * rp + R[1];
      points[idy + 2] = az[j] * rp + R[2];
      weights[aux] = aw[j] * rw;
    }
  }
}

/* ---------------------------------------------------------------- Becke */
/* src/utils/utils.cpp:35-43 */
static double dist(const double *a, const double *b) {
  double out = 0.0;
  for (int i = 0; i < 3; ++i) {
    double aux = a[i] - b[i];
    out += aux * aux;
  }
  return sqrt(out);
}

/* src/grid/becke.cpp:79-176.  `offsets` (ncenter+1) gives each atom's first
 * point; with equal atomic grids it equals atom * (size / ncenter) as in the
 * reference.  Parallel over points (the reference parallelises the same loop). */
void orc_becke_weights(int ncenter, int size, const double *radii, const double *origin,
                       const double *points, const int *offsets, double *becke) {
  int asize = (ncenter * (ncenter + 1)) / 2;
  double *R_ij = (double *)malloc(sizeof(double) * asize);
  double *a_ij = (double *)malloc(sizeof(double) * asize);
  int offset = 0;
  for (int i = 0; i < ncenter; i++)
    for (int j = 0; j <= i; j++) R_ij[offset++] = dist(&origin[3 * i], &origin[3 * j]);
  offset = 0;
  for (int i = 0; i < ncenter; i++)
    for (int j = 0; j <= i; j++) {
      double aux = (radii[i] - radii[j]) / (radii[i] + radii[j]);
      aux = aux / (aux * aux - 1.0);
      if (aux > 0.45) aux = 0.45;
      else if (aux < -0.45) aux = -0.45;
      a_ij[offset++] = aux;
    }
  unsigned int order = 3;
  for (int atom = 0; atom < ncenter; ++atom) {
    int npoint = offsets[atom + 1] - offsets[atom];
#pragma omp parallel for schedule(static)
    for (int point = 0; point < npoint; ++point) {
      double sum = 0.0, aux = 0.0;
      unsigned int idx = (offsets[atom] + point) * 3;
      for (int i = 0; i < ncenter; ++i) {
        double p = 1.0;
        for (int j = 0; j < ncenter; ++j) {
          if (i == j) continue;
          int off = (i < j) ? (j * (j + 1)) / 2 + i : (i * (i + 1)) / 2 + j;
          double r_i = dist(&points[idx], &origin[i * 3]);
          double r_j = dist(&points[idx], &origin[j * 3]);
          double mu = (r_i - r_j) / R_ij[off];
          double s = mu + a_ij[off] * ((1.0 - 2 * (i < j)) * (1.0 - mu * mu));
          for (unsigned int k = 1; k <= order; k++) s = 0.5 * s * (3 - s * s);
          s = 0.5 * (1.0 - s);
          p *= s;
        }
        if (i == atom) aux = p;
        sum += p;
      }
      becke[offsets[atom] + point] = aux / sum;
    }
  }
  free(R_ij);
  free(a_ij);
}

/* ------------------------------------------------------------------ GTO */
static int fact2(int n) {
  if (n < 1) return 0;
  int o = 1;
  for (int i = n; i > 0; i -= 2) o *= i;
  return o;
}

/* src/system/gto.cpp:29-39 */
double orc_prim_norm(const int *l, double zeta) {
  int aux = l[0] + l[1] + l[2];
  return (pow((2.0 * zeta / M_PI), 0.75)) /
         sqrt(fact2(abs(2 * l[0] - 1)) * fact2(abs(2 * l[1] - 1)) * fact2(abs(2 * l[2] - 1)) /
              (pow((4.0 * zeta), aux)));
}

/* src/ints/overlap.cpp:12-138: Obara-Saika overlap of two primitives. */
static void os_recursion(double *x, double *y, double *z, const double *PA, const double *PB,
                         double gamma, int l_a, int l_b, int max_l) {
  double pp = 1.0 / (2.0 * gamma);
  x[0] = 1.0; y[0] = 1.0; z[0] = 1.0;
  x[1] = PB[0]; y[1] = PB[1]; z[1] = PB[2];
  for (int j = 1; j < l_b; j++) {
    int idx = j;
    x[idx + 1] = PB[0] * x[j] + j * pp * x[idx - 1];
    y[idx + 1] = PB[1] * y[j] + j * pp * y[idx - 1];
    z[idx + 1] = PB[2] * z[j] + j * pp * z[idx - 1];
  }
  x[max_l] = PA[0]; y[max_l] = PA[1]; z[max_l] = PA[2];
  for (int j = 1; j <= l_b; j++) {
    int idx = max_l + j;
    x[idx] = PA[0] * x[j] + j * pp * x[j - 1];
    y[idx] = PA[1] * y[j] + j * pp * y[j - 1];
    z[idx] = PA[2] * z[j] + j * pp * z[j - 1];
  }
  for (int i = 1; i < l_a; i++) {
    int idx = i * max_l, idxp1 = (i + 1) * max_l, idxm1 = (i - 1) * max_l;
    x[idxp1] = PA[0] * x[idx] + i * pp * x[idxm1];
    y[idxp1] = PA[1] * y[idx] + i * pp * y[idxm1];
    z[idxp1] = PA[2] * z[idx] + i * pp * z[idxm1];
    for (int j = 1; j <= l_b; j++) {
      idx++; idxp1++; idxm1++;
      x[idxp1] = PA[0] * x[idx] + i * pp * x[idxm1] + j * pp * x[idx - 1];
      y[idxp1] = PA[1] * y[idx] + i * pp * y[idxm1] + j * pp * y[idx - 1];
      z[idxp1] = PA[2] * z[idx] + i * pp * z[idxm1] + j * pp * z[idx - 1];
    }
  }
}

double orc_overlap_prim(const int *la, const double *A, double za, double ca, double na,
                        const int *lb, const double *B, double zb, double cb, double nb) {
  double gamma = za + zb, gi = 1.0 / gamma, PA[3], PB[3], AB2 = 0.0;
  int Ia = 0, Ib = 0;
  for (int i = 0; i < 3; ++i) {
    double AB = A[i] - B[i];
    double P0 = (za * A[i] + zb * B[i]) * gi;
    PA[i] = P0 - A[i];
    PB[i] = P0 - B[i];
    AB2 += AB * AB;
    Ia += la[i];
    Ib += lb[i];
  }
  double pre = exp(-za * zb * AB2 * gi) * (sqrt(M_PI * gi) * M_PI * gi * ca * cb * na * nb);
  int max_l = (Ia > Ib ? Ia : Ib) + 4;
  double *x = calloc(max_l * max_l, sizeof(double));
  double *y = calloc(max_l * max_l, sizeof(double));
  double *z = calloc(max_l * max_l, sizeof(double));
  os_recursion(x, y, z, PA, PB, gamma, Ia + 2, Ib + 2, max_l);
  double out = pre * x[la[0] * max_l + lb[0]] * y[la[1] * max_l + lb[1]] *
               z[la[2] * max_l + lb[2]];
  free(x); free(y); free(z);
  return out;
}

/* Basis evaluation (src/system/gto.cpp:41-51,180-192; basis_set.cpp:69-82).
 * Functions are described by flat arrays: for function f, l[3f..3f+2],
 * origin[3f..], nprim[f], first prim off[f]; per primitive zeta, coeff.
 * Writes phi[p * nf + f] (point-major, as BasisSet_compute does). */
void orc_basis_compute(int nf, const int *l, const double *origin, const int *nprim,
                       const int *off, const double *zeta, const double *coeff,
                       int npoint, const double *r, double *phi) {
  /* per-primitive and per-contraction norms */
  int ntot = 0;
  for (int f = 0; f < nf; ++f) ntot += nprim[f];
  double *pn = malloc(sizeof(double) * ntot), *cn = malloc(sizeof(double) * nf);
  for (int f = 0; f < nf; ++f) {
    for (int k = 0; k < nprim[f]; ++k) pn[off[f] + k] = orc_prim_norm(&l[3 * f], zeta[off[f] + k]);
    double s = 0.0;
    for (int a = 0; a < nprim[f]; ++a)
      for (int b = 0; b < nprim[f]; ++b)
        s += orc_overlap_prim(&l[3 * f], &origin[3 * f], zeta[off[f] + a], coeff[off[f] + a],
                              pn[off[f] + a], &l[3 * f], &origin[3 * f], zeta[off[f] + b],
                              coeff[off[f] + b], pn[off[f] + b]);
    cn[f] = 1.0 / sqrt(s * 1.0 * 1.0);
  }
#pragma omp parallel for schedule(static)
  for (int p = 0; p < npoint; ++p) {
    const double *rp = &r[3 * p];
    for (int f = 0; f < nf; ++f) {
      double out = 0.0;
      for (int k = 0; k < nprim[f]; ++k) {
        double RP2 = 0.0, factor = 1.0;
        for (int i = 0; i < 3; ++i) {
          double aux = rp[i] - origin[3 * f + i];
          factor *= pow(aux, l[3 * f + i]);
          RP2 += aux * aux;
        }
        out += coeff[off[f] + k] * pn[off[f] + k] * factor * exp(-zeta[off[f] + k] * RP2);
      }
      phi[(long)p * nf + f] = out * cn[f];
    }
  }
  free(pn);
  free(cn);
}

/* ---------------------------------------------------------- quadratures */
/* rho[p] = sum_ij D_ij phi_i phi_j (the density the reference drivers form
 * point by point, psi_hybrid.py:144-150: sum_i phi_i (D phi)_i).  phi [n][N]. */
void orc_density(int n, int N, const double *phi, const double *D, double *rho) {
#pragma omp parallel for schedule(static)
  for (int p = 0; p < N; ++p) {
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
      double t = 0.0;
      for (int j = 0; j < n; ++j) t += D[i * n + j] * phi[(long)j * N + p];
      acc += phi[(long)i * N + p] * t;
    }
    rho[p] = acc;
  }
}

/* F_ij = sum_p (phi_i phi_j C)_p bw_p w_p for i <= j, mirrored
 * (src/wavefunction/nwavefunction.cpp:77-107,161-197 with
 * BeckeGrid::integrate, becke.cpp:178-191), streamed instead of
 * materialising Psi[n(n+1)/2][N]. */
void orc_quadrature(int n, int N, const double *phi, const double *C, const double *bw,
                    const double *w, double *F) {
  int npair = n * (n + 1) / 2;
#pragma omp parallel for schedule(dynamic, 8)
  for (int e = 0; e < npair; ++e) {
    int i = 0, rem = e;
    while (rem >= n - i) { rem -= n - i; ++i; }
    int j = i + rem;
    const double *a = phi + (long)i * N, *b = phi + (long)j * N;
    double s = 0.0;
    for (int p = 0; p < N; ++p) s += a[p] * b[p] * C[p] * bw[p] * w[p];
    F[i * n + j] = s;
    F[j * n + i] = s;
  }
}

/* ------------------------------------------------- moments / projection */
/* src/horton/moments.cpp:59-125 */
static void pure_poly(double *output, long lmax) {
  if (lmax <= 1) return;
  double z = output[0], x = output[1], y = output[2];
  double r2 = x * x + y * y + z * z;
  double *pi_old = malloc(sizeof(double) * (lmax + 1)), *pi_new = malloc(sizeof(double) * (lmax + 1));
  double *a = malloc(sizeof(double) * (lmax + 1)), *b = malloc(sizeof(double) * (lmax + 1));
  pi_old[0] = 1; pi_new[0] = z; pi_new[1] = 1; a[1] = x; b[1] = y;
  int old_offset = 0, old_npure = 3;
  for (int l = 2; l <= lmax; l++) {
    int new_npure = old_npure + 2, new_offset = old_offset + old_npure;
    double factor = (2 * l - 1);
    for (int m = 0; m <= l - 2; m++) {
      double tmp = pi_old[m];
      pi_old[m] = pi_new[m];
      pi_new[m] = (z * factor * pi_old[m] - r2 * (l + m - 1) * tmp) / (l - m);
    }
    pi_old[l - 1] = pi_new[l - 1];
    pi_new[l] = factor * pi_old[l - 1];
    pi_new[l - 1] = z * pi_new[l];
    a[l] = x * a[l - 1] - y * b[l - 1];
    b[l] = x * b[l - 1] + y * a[l - 1];
    output[new_offset] = pi_new[0];
    factor = M_SQRT2;
    for (int m = 1; m <= l; m++) {
      factor /= sqrt((l + m) * (l - m + 1));
      output[new_offset + 2 * m - 1] = factor * a[m] * pi_new[m];
      output[new_offset + 2 * m] = factor * b[m] * pi_new[m];
    }
    old_npure = new_npure;
    old_offset = new_offset;
  }
  free(pi_old); free(pi_new); free(a); free(b);
}

/* AtomicGrid::spherical_expansion (src/grid/atomic_grid.cpp:82-136) with
 * dot_multi_moments mtype 4 (src/horton/dot_multi.cpp:148-185): f is the
 * function on the atomic grid, out[nrad][lsize]. */
void orc_spherical_expansion(int nrad, int nang, const double *points, const double *weights,
                             const double *center, const double *f, int lmax, double *out) {
  int lsize = (lmax + 1) * (lmax + 1);
  double *work = malloc(sizeof(double) * (lsize + 3));
  memset(out, 0, sizeof(double) * nrad * lsize);
  for (int i = 0; i < nrad; ++i) {
    double *o = out + (long)i * lsize;
    for (int j = 0; j < nang; ++j) {
      long p = (long)i * nang + j;
      double term = f[p] * weights[p];
      o[0] += term;
      if (lmax > 0) {
        double d0 = points[3 * p] - center[0], d1 = points[3 * p + 1] - center[1],
               d2 = points[3 * p + 2] - center[2];
        double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        work[0] = d2 / r; work[1] = d0 / r; work[2] = d1 / r;
        pure_poly(work, lmax);
        for (int m = 1; m < lsize; m++) o[m] += term * work[m - 1];
      }
    }
  }
  for (int i = 0; i < nrad; ++i) {
    double sigma = 0.0;
    for (int j = 0; j < nang; ++j) sigma += weights[(long)i * nang + j];
    for (int m = 0; m < lsize; ++m) out[(long)i * lsize + m] /= sigma;
  }
  int c = 0;
  for (int l = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m, ++c)
      for (int i = 0; i < nrad; ++i) out[(long)i * lsize + c] *= sqrt(4.0 * M_PI * (2.0 * l + 1));
  free(work);
}

/* --------------------------------------------------------------- splines */
/* src/horton/cubic_spline.cpp:54-103 */
void orc_tridiagsym_solve(double *diag_mid, double *diag_up, double *right, double *solution,
                          int n) {
  double denominator, tmp1, tmp2;
  tmp1 = diag_up[0];
  tmp2 = 0.0;
  diag_up[0] /= diag_mid[0];
  right[0] /= diag_mid[0];
  for (int i = 1; i < n; i++) {
    denominator = (diag_mid[i] - diag_up[i - 1] * tmp1);
    if (i < n - 1) {
      tmp2 = diag_up[i];
      diag_up[i] /= denominator;
    }
    right[i] = (right[i] - right[i - 1] * tmp1) / denominator;
    tmp1 = tmp2;
  }
  solution[n - 1] = right[n - 1];
  for (int i = n - 2; i >= 0; i--) solution[i] = right[i] - diag_up[i] * solution[i + 1];
}

void orc_spline_dt(const double *y, double *dt, int n) {
  double *mid = malloc(sizeof(double) * n), *up = malloc(sizeof(double) * n),
         *right = malloc(sizeof(double) * n);
  mid[0] = 2.0; up[0] = 1.0; right[0] = 3.0 * (y[1] - y[0]);
  for (int i = 1; i < n - 1; i++) {
    mid[i] = 4.0; up[i] = 1.0; right[i] = 3.0 * (y[i + 1] - y[i - 1]);
  }
  mid[n - 1] = 2.0;
  right[n - 1] = 3.0 * (y[n - 1] - y[n - 2]);
  orc_tridiagsym_solve(mid, up, right, dt, n);
  free(mid); free(up); free(right);
}

/* orc_spherical_expansion of k functions f[c * ld + p] of one atom's points
 * (same arithmetic per function), out [k][nrad][lsize]; OpenMP over functions. */
void orc_spherical_expansion_many(int nrad, int nang, const double *points, const double *weights,
                                  const double *center, int k, const double *f, long ld, int lmax,
                                  double *out) {
  const long lsize = (long)(lmax + 1) * (lmax + 1);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < k; ++c)
    orc_spherical_expansion(nrad, nang, points, weights, center, f + (long)c * ld, lmax,
                            out + (long)c * nrad * lsize);
}

/* orc_spline_dt of ncol columns y[c * n + i]; OpenMP over columns. */
void orc_spline_dt_many(const double *y, double *dt, int n, int ncol) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < ncol; ++c) orc_spline_dt(y + (long)c * n, dt + (long)c * n, n);
}

/* ----------------------------------------------------------- FEM (ODE) */
/* Cubic Hermite FEM assembly (src/horton/ode2.cpp:232-321).  The segment
 * integrals of products of Hermite basis polynomials are evaluated exactly
 * here by integrating monomials (the reference tabulates the same rationals). */
static const double HP[4][4] = {{1, 0, -3, 2}, {0, 1, -2, 1}, {0, 0, 3, -2}, {0, 0, -1, 1}};

static int seg_piece(long c, long k, long g) {
  if (c == g) return (int)k;
  if (c == g + 1) return (int)(2 + k);
  return -1;
}

static void poly_of(int piece, int deriv, double *o) {
  for (int i = 0; i < 4; ++i) o[i] = 0.0;
  if (piece < 0) return;
  if (!deriv) for (int i = 0; i < 4; ++i) o[i] = HP[piece][i];
  else { o[0] = HP[piece][1]; o[1] = 2 * HP[piece][2]; o[2] = 3 * HP[piece][3]; }
}

static double seg_integral(const int *pieces, const int *derivs, int nfac) {
  double acc[10] = {1, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  int deg = 0;
  for (int f = 0; f < nfac; ++f) {
    double q[4], nxt[10] = {0};
    poly_of(pieces[f], derivs[f], q);
    for (int i = 0; i <= deg; ++i)
      for (int j = 0; j < 4; ++j) nxt[i + j] += acc[i] * q[j];
    deg += 3;
    memcpy(acc, nxt, sizeof(acc));
  }
  long num = 0;
  for (int k = 0; k <= deg; ++k) num += (long)acc[k] * (2520 / (k + 1));
  return (double)num / 2520.0;
}

static double ov(long xmax, int nfac, const long *idx, const int *der) {
  long c0 = idx[0] / 2;
  for (int f = 1; f < nfac; ++f) if (labs(idx[f] / 2 - c0) >= 2) return 0.0;
  double result = 0.0;
  for (int side = 0; side < 2; ++side) {
    long g = side == 0 ? c0 - 1 : c0;
    int ok = side == 0 ? (c0 >= 1 && c0 <= xmax) : (c0 >= 0 && c0 <= xmax - 1);
    if (!ok) continue;
    int pieces[3];
    for (int f = 0; f < nfac; ++f) pieces[f] = seg_piece(idx[f] / 2, idx[f] % 2, g);
    result += seg_integral(pieces, der, nfac);
  }
  return result;
}

static double node(long x, long c, long k, int d) { return (k == d) ? (double)(x == c) : 0.0; }

void orc_build_ode2(const double *b, const double *a, const double *f, const double *bcs,
                    double *coeffs, double *rhs, long npoint) {
  long nfn = 2 * npoint, skiprow[2] = {-1, -1};
  int counter = 0;
  if (bcs[0] == bcs[0]) { coeffs[0] = 1; rhs[0] = bcs[0]; skiprow[counter++] = 0; }
  if (bcs[1] == bcs[1]) { coeffs[nfn + 1] = 1; rhs[1] = bcs[1]; if (counter < 2) skiprow[counter] = 1; counter++; }
  if (bcs[2] == bcs[2]) { coeffs[nfn * (nfn - 1) - 2] = 1; rhs[nfn - 2] = bcs[2]; if (counter < 2) skiprow[counter] = nfn - 2; counter++; }
  if (bcs[3] == bcs[3]) { coeffs[nfn * nfn - 1] = 1; rhs[nfn - 1] = bcs[3]; if (counter < 2) skiprow[counter] = nfn - 1; counter++; }
  long xmax = npoint - 1;
  for (long irow = 0; irow < nfn; irow++) {
    if (irow == skiprow[0] || irow == skiprow[1]) continue;
    long begin = 2 * (irow / 2 - 1), end = 2 * (irow / 2 + 2);
    if (begin < 0) begin = 0;
    if (end > nfn) end = nfn;
    for (long icol = begin; icol < end; icol++) {
      double *coeff = coeffs + (irow * nfn + icol);
      long i2[2] = {irow, icol};
      int d2[2] = {1, 1};
      *coeff -= ov(xmax, 2, i2, d2);
      for (long ifoo = begin; ifoo < end; ifoo++) {
        long i3[3] = {irow, icol, ifoo};
        if (b[ifoo] != 0) { int d3[3] = {0, 1, 0}; *coeff += b[ifoo] * ov(xmax, 3, i3, d3); }
        if (a[ifoo] != 0) { int d3[3] = {0, 0, 0}; *coeff += a[ifoo] * ov(xmax, 3, i3, d3); }
      }
      *coeff += node(npoint - 1, irow / 2, irow % 2, 0) * node(npoint - 1, icol / 2, icol % 2, 1);
      *coeff -= node(0, irow / 2, irow % 2, 0) * node(0, icol / 2, icol % 2, 1);
    }
    for (long ifoo = begin; ifoo < end; ifoo++) {
      if (f[ifoo] != 0) {
        long i2[2] = {irow, ifoo};
        int d2[2] = {0, 0};
        rhs[irow] += f[ifoo] * ov(xmax, 2, i2, d2);
      }
    }
  }
}

/* ------------------------------------------------- potential evaluation */
/* eval_decomposition_grid (src/horton/evaluate.cpp:129-220) for splines with
 * PotentialExtrapolation (extrapolation.cpp:149-183) on a Chebyshev (kind 0,
 * p0 = radii) or Power (kind 1, p0 = rmin, p1 = power) transform.
 * y, dt: [nspline][n]; output += at every point. */
void orc_eval_decomposition(int kind, double p0, double p1, int n, int nspline, const double *y,
                            const double *dt, const double *center, int npoint,
                            const double *points, double *output) {
  long lmax = (long)sqrt((double)nspline) - 1;
  double first_x, last_x;
  if (kind == 0) { first_x = orc_cheb_radius(p0, n, 0); last_x = orc_cheb_radius(p0, n, n - 1); }
  else { first_x = orc_power_radius(p0, p1, 0); last_x = orc_power_radius(p0, p1, n - 1); }
  double *amp_l = malloc(sizeof(double) * nspline), *amp_r = malloc(sizeof(double) * nspline);
  int *ls = malloc(sizeof(int) * nspline);
  for (int l = 0, c = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m, ++c) {
      ls[c] = l;
      amp_l[c] = y[(long)c * n] / pow(first_x, l);
      amp_r[c] = y[(long)c * n + n - 1] * pow(last_x, l + 1);
    }
#pragma omp parallel
  {
    double *work = malloc(sizeof(double) * (nspline + 3));
#pragma omp for schedule(static)
    for (int i = 0; i < npoint; ++i) {
      double x = points[3 * i] - center[0], yy = points[3 * i + 1] - center[1],
             z = points[3 * i + 2] - center[2];
      double d = sqrt(x * x + yy * yy + z * z);
      double t = 0.0, u = 0.0;
      int j = 0;
      if (d >= first_x && d <= last_x) {
        t = kind == 0 ? orc_cheb_inv(p0, n, d) : pow(d / p0, 1.0 / p1) - 1;
        j = (int)floor(t);
        if (j == n - 1) j = n - 2;
        if (j < 0) j = 0;
        u = t - j;
      }
      for (int c = 0; c < nspline; ++c) {
        double s;
        if (d < first_x) s = amp_l[c] * pow(d, ls[c]);
        else if (d <= last_x) {
          const double *Y = y + (long)c * n, *D = dt + (long)c * n;
          double zz = Y[j + 1] - Y[j];
          s = Y[j] + u * (D[j] + u * (3 * zz - 2 * D[j] - D[j + 1] + u * (-2 * zz + D[j] + D[j + 1])));
        } else s = amp_r[c] / pow(d, ls[c] + 1);
        work[c] = s;  /* spline values first, combined below */
      }
      double acc = output[i];
      acc += work[0] * 0.28209479177387814347;
      if (lmax > 0) {
        double *sh = malloc(sizeof(double) * (nspline + 3));
        sh[0] = z; sh[1] = x; sh[2] = yy;
        if (lmax > 1) pure_poly(sh, lmax);
        long counter = 0;
        double dpowl = 1.0;
        for (long l = 1; l <= lmax; l++) {
          dpowl = dpowl / d;
          double factor = sqrt(2 * l + 1);
          for (long m = -l; m <= l; m++) {
            acc += work[counter + 1] * factor * 0.28209479177387814347 * dpowl * sh[counter];
            counter++;
          }
        }
        free(sh);
      }
      output[i] = acc;
    }
    free(work);
  }
  free(amp_l); free(amp_r); free(ls);
}

/* orc_eval_decomposition for k sets of splines on the same atom (y, dt:
 * [k][nspline][n]; output row c at output + c * ldo): the point's distance,
 * spline interval and harmonics are computed once and shared; each set's
 * arithmetic is that of orc_eval_decomposition, so every row equals a
 * separate call bit for bit. */
void orc_eval_decomposition_many(int kind, double p0, double p1, int n, int nspline, int k,
                                 const double *y, const double *dt, const double *center,
                                 int npoint, const double *points, double *output, long ldo) {
  long lmax = (long)sqrt((double)nspline) - 1;
  double first_x, last_x;
  if (kind == 0) { first_x = orc_cheb_radius(p0, n, 0); last_x = orc_cheb_radius(p0, n, n - 1); }
  else { first_x = orc_power_radius(p0, p1, 0); last_x = orc_power_radius(p0, p1, n - 1); }
  const long ks = (long)nspline * n;
  double *amp_l = malloc(sizeof(double) * nspline * k), *amp_r = malloc(sizeof(double) * nspline * k);
  int *ls = malloc(sizeof(int) * nspline);
  for (int l = 0, c = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m, ++c) ls[c] = l;
  for (int b = 0; b < k; ++b)
    for (int c = 0; c < nspline; ++c) {
      amp_l[b * nspline + c] = y[b * ks + (long)c * n] / pow(first_x, ls[c]);
      amp_r[b * nspline + c] = y[b * ks + (long)c * n + n - 1] * pow(last_x, ls[c] + 1);
    }
#pragma omp parallel
  {
    double *work = malloc(sizeof(double) * (nspline + 3));
    double *sh = malloc(sizeof(double) * (nspline + 3));
    double *fac = malloc(sizeof(double) * (nspline + 3));
#pragma omp for schedule(static)
    for (int i = 0; i < npoint; ++i) {
      double x = points[3 * i] - center[0], yy = points[3 * i + 1] - center[1],
             z = points[3 * i + 2] - center[2];
      double d = sqrt(x * x + yy * yy + z * z);
      double t = 0.0, u = 0.0;
      int j = 0;
      if (d >= first_x && d <= last_x) {
        t = kind == 0 ? orc_cheb_inv(p0, n, d) : pow(d / p0, 1.0 / p1) - 1;
        j = (int)floor(t);
        if (j == n - 1) j = n - 2;
        if (j < 0) j = 0;
        u = t - j;
      }
      if (lmax > 0) {
        sh[0] = z; sh[1] = x; sh[2] = yy;
        if (lmax > 1) pure_poly(sh, lmax);
        long counter = 0;
        double dpowl = 1.0;
        for (long l = 1; l <= lmax; l++) {
          dpowl = dpowl / d;
          double factor = sqrt(2 * l + 1);
          for (long m = -l; m <= l; m++) fac[counter++] = factor * 0.28209479177387814347 * dpowl;
        }
      }
      for (int b = 0; b < k; ++b) {
        const double *yb = y + b * ks, *db = dt + b * ks;
        for (int c = 0; c < nspline; ++c) {
          double s;
          if (d < first_x) s = amp_l[b * nspline + c] * pow(d, ls[c]);
          else if (d <= last_x) {
            const double *Y = yb + (long)c * n, *D = db + (long)c * n;
            double zz = Y[j + 1] - Y[j];
            s = Y[j] + u * (D[j] + u * (3 * zz - 2 * D[j] - D[j + 1] + u * (-2 * zz + D[j] + D[j + 1])));
          } else s = amp_r[b * nspline + c] / pow(d, ls[c] + 1);
          work[c] = s;
        }
        double acc = output[b * ldo + i];
        acc += work[0] * 0.28209479177387814347;
        for (long c = 0; c + 1 < nspline; ++c) acc += work[c + 1] * fac[c] * sh[c];
        output[b * ldo + i] = acc;
      }
    }
    free(work); free(sh); free(fac);
  }
  free(amp_l); free(amp_r); free(ls);
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
