// Real regular solid harmonics S_lm(x, y, z) for l = 2..lmax, used by the
// Lebedev projection and by the multipole evaluation of the Poisson
// potential.  Input out[0..2] = (z, x, y) (the l = 1 block), output out[3..]
// holds l = 2..lmax, each l as m = 0, (cos 1, sin 1), ..., (cos l, sin l).
//
// Recursion (Helgaker, Jorgensen & Olsen, "Molecular Electronic-Structure
// Theory", sec. 6.4): the z/r-polynomials Pi_l^m obey
//   Pi_l^m = [(2l-1) z Pi_{l-1}^m - (l+m-1) r^2 Pi_{l-2}^m] / (l-m),
//   Pi_l^l = (2l-1) Pi_{l-1}^{l-1},  Pi_l^{l-1} = z Pi_l^l,
// the azimuthal factors obey C_l + i S_l = (x + i y)(C_{l-1} + i S_{l-1}), and
// the normalisation is sqrt(2 (l-m)!/(l+m)!).  The ordering, normalisation and
// operation order are those of nAPMO (src/horton/moments.cpp:59-125), so
// host results are bit-identical to the reference.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define NAPMO_HD __host__ __device__ __forceinline__
#else
#define NAPMO_HD inline
#endif

namespace napmo {

constexpr int kMaxLmax = 40;

NAPMO_HD void solid_harmonics(double *out, long lmax) {
  if (lmax <= 1) return;
  const double z = out[0];
  const double x = out[1];
  const double y = out[2];
  const double r2 = x * x + y * y + z * z;
  double pold[kMaxLmax + 1], pnew[kMaxLmax + 1];
  double cs[kMaxLmax + 1], sn[kMaxLmax + 1];
  pold[0] = 1;
  pnew[0] = z;
  pnew[1] = 1;
  cs[1] = x;
  sn[1] = y;
  long prev_off = 0, prev_n = 3;
  for (long l = 2; l <= lmax; l++) {
    const long off = prev_off + prev_n;
    double fac = (2 * l - 1);
    for (long m = 0; m <= l - 2; m++) {
      const double keep = pold[m];
      pold[m] = pnew[m];
      pnew[m] = (z * fac * pold[m] - r2 * (l + m - 1) * keep) / (l - m);
    }
    pold[l - 1] = pnew[l - 1];
    pnew[l] = fac * pold[l - 1];
    pnew[l - 1] = z * pnew[l];
    cs[l] = x * cs[l - 1] - y * sn[l - 1];
    sn[l] = x * sn[l - 1] + y * cs[l - 1];
    out[off] = pnew[0];
    fac = M_SQRT2;
    for (long m = 1; m <= l; m++) {
      fac /= sqrt((double)((l + m) * (l - m + 1)));
      out[off + 2 * m - 1] = fac * cs[m] * pnew[m];
      out[off + 2 * m] = fac * sn[m] * pnew[m];
    }
    prev_n += 2;
    prev_off = off;
  }
}

}  // namespace napmo
