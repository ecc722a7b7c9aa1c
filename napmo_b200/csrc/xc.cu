// Local functionals on the grid, elementwise on the device:
//
//   LDA (nAPMO's Functional 'lda': LibXC lda_x + lda_c_vwn, unpolarised,
//   napmo/functional/xc_interface.py:29-90), in the published forms that
//   LibXC evaluates:
//     Dirac-Slater exchange  e_x = 3/4 CX rho^(1/3),  v_x = CX rho^(1/3),
//                            CX = -(3/pi)^(1/3)
//     VWN5 correlation       (Vosko, Wilk, Nusair, Can. J. Phys. 58, 1200
//                            (1980), paramagnetic fit), x = sqrt(r_s):
//       e_c = A [ln(x^2/X) + 2b/Q atan(Q/(2x+b))
//                - b x0/X(x0) (ln((x-x0)^2/X) + 2(b+2x0)/Q atan(Q/(2x+b)))]
//       v_c = e_c - x/6 de_c/dx
//     with A = 0.0310907, b = 3.72744, c = 12.9352, x0 = -0.10498,
//     X = x^2 + b x + c, Q = sqrt(4c - b^2).  Densities below 1e-24 give 0
//     (nAPMO's LibXC fixtures place the cut between 3.1e-25 and 1.2e-22).
//
//   epc17-2 electron-proton correlation at common points
//   (napmo/functional/interspecies_correlation.py:36-68): energy per electron
//   -rho_N / den, den = a - b sqrt(rho_E rho_N) + c rho_E rho_N with
//   (a, b, c) = (2.35, 2.4, 6.6), and the potentials of both species; when any
//   density of the call is below 1e-200 every point uses the alternative
//   potentials, as nAPMO does (a device flag set by a first pass).  Negative
//   densities (rounding) count as zero.
#include <cuda_runtime.h>

#include <cmath>

#include "capi_common.cuh"

namespace napmo {
namespace {

constexpr double kDensCut = 1e-24;
constexpr double kVwnA = 0.0310907, kVwnB = 3.72744, kVwnC = 12.9352, kVwnX0 = -0.10498;

__global__ void lda_xc_kernel(long n, const double *__restrict__ rho, double *__restrict__ xzk,
                              double *__restrict__ xv, double *__restrict__ czk,
                              double *__restrict__ cv) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r = rho[i];
  const bool on = r >= kDensCut;
  if (xzk || xv) {
    const double cx = -cbrt(3.0 / M_PI);
    const double r13 = on ? cbrt(r) : 0.0;
    if (xzk) xzk[i] = on ? 0.75 * cx * r13 : 0.0;
    if (xv) xv[i] = on ? cx * r13 : 0.0;
  }
  if (czk || cv) {
    double ec = 0.0, vc = 0.0;
    if (on) {
      const double b = kVwnB, c = kVwnC, x0 = kVwnX0;
      const double x = sqrt(cbrt(3.0 / (4.0 * M_PI * r)));
      const double X = x * x + b * x + c;
      const double X0 = x0 * x0 + b * x0 + c;
      const double Q = sqrt(4.0 * c - b * b);
      const double at = atan(Q / (2.0 * x + b));
      ec = kVwnA * (log(x * x / X) + 2.0 * b / Q * at -
                    b * x0 / X0 * (log((x - x0) * (x - x0) / X) + 2.0 * (b + 2.0 * x0) / Q * at));
      const double dX = 2.0 * x + b;
      const double den = dX * dX + Q * Q;
      const double dec = kVwnA * (2.0 / x - dX / X - 4.0 * b / den -
                                  b * x0 / X0 * (2.0 / (x - x0) - dX / X - 4.0 * (b + 2.0 * x0) / den));
      vc = ec - x / 6.0 * dec;
    }
    if (czk) czk[i] = ec;
    if (cv) cv[i] = vc;
  }
}

// Spin-polarised LDA (nAPMO's DFT with spin 'polarized' for open shells,
// dft_solver.py:35, LibXC lda_x and lda_c_vwn with two spin densities):
//   exchange  e_x = -3/4 (6/pi)^(1/3) (rho_a^(4/3) + rho_b^(4/3)),
//             v_s = -(6 rho_s / pi)^(1/3);
//   VWN5      e_c(r_s, z) = e_P + a_c f(z) / f''(0) (1 - z^4)
//                         + (e_F - e_P) f(z) z^4,  z = (rho_a - rho_b) / rho,
//             f(z) = ((1+z)^(4/3) + (1-z)^(4/3) - 2) / (2^(4/3) - 2),
//             v_s = e_c - (r_s / 3) de_c/dr_s + (s - z) de_c/dz (s = +1, -1),
//   with the paramagnetic (P), ferromagnetic (F) and spin-stiffness (a_c)
//   fits of Vosko, Wilk and Nusair.  zk are energies per particle of the
//   total density; zero where rho_a + rho_b < 1e-24, negative spin
//   densities counting as zero.
constexpr double kVwnFA = 0.01554535, kVwnFB = 7.06042, kVwnFC = 18.0578, kVwnFX0 = -0.32500;
constexpr double kVwnAB = 1.13107, kVwnAC = 13.0045, kVwnAX0 = -0.0047584;

__device__ __forceinline__ void vwn_fit(double x, double A, double b, double c, double x0,
                                        double &g, double &dg) {
  const double X = x * x + b * x + c;
  const double X0 = x0 * x0 + b * x0 + c;
  const double Q = sqrt(4.0 * c - b * b);
  const double at = atan(Q / (2.0 * x + b));
  g = A * (log(x * x / X) + 2.0 * b / Q * at -
           b * x0 / X0 * (log((x - x0) * (x - x0) / X) + 2.0 * (b + 2.0 * x0) / Q * at));
  const double dX = 2.0 * x + b;
  const double den = dX * dX + Q * Q;
  dg = A * (2.0 / x - dX / X - 4.0 * b / den -
            b * x0 / X0 * (2.0 / (x - x0) - dX / X - 4.0 * (b + 2.0 * x0) / den));
}

__global__ void lda_xc_pol_kernel(long n, const double *__restrict__ rho_a,
                                  const double *__restrict__ rho_b, double *__restrict__ xzk,
                                  double *__restrict__ xva, double *__restrict__ xvb,
                                  double *__restrict__ czk, double *__restrict__ cva,
                                  double *__restrict__ cvb) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double ra = fmax(rho_a[i], 0.0), rb = fmax(rho_b[i], 0.0);
  const double rho = ra + rb;
  const bool on = rho >= kDensCut;
  if (xzk || xva || xvb) {
    const double c = -cbrt(6.0 / M_PI);
    const double a13 = cbrt(ra), b13 = cbrt(rb);
    if (xzk) xzk[i] = on ? 0.75 * c * (ra * a13 + rb * b13) / rho : 0.0;
    if (xva) xva[i] = on ? c * a13 : 0.0;
    if (xvb) xvb[i] = on ? c * b13 : 0.0;
  }
  if (czk || cva || cvb) {
    double ec = 0.0, va = 0.0, vb = 0.0;
    if (on) {
      const double z = fmin(fmax((ra - rb) / rho, -1.0), 1.0);
      const double x = sqrt(cbrt(3.0 / (4.0 * M_PI * rho)));
      double eP, dP, eF, dF, ac, dac;
      vwn_fit(x, kVwnA, kVwnB, kVwnC, kVwnX0, eP, dP);
      vwn_fit(x, kVwnFA, kVwnFB, kVwnFC, kVwnFX0, eF, dF);
      vwn_fit(x, -1.0 / (6.0 * M_PI * M_PI), kVwnAB, kVwnAC, kVwnAX0, ac, dac);
      const double fden = exp2(4.0 / 3.0) - 2.0;
      const double fpp = 4.0 / (9.0 * (cbrt(2.0) - 1.0));
      const double zp = cbrt(1.0 + z), zm = cbrt(1.0 - z);
      const double f = ((1.0 + z) * zp + (1.0 - z) * zm - 2.0) / fden;
      const double df = (4.0 / 3.0) * (zp - zm) / fden;
      const double z3 = z * z * z, z4 = z3 * z;
      ec = eP + ac * f / fpp * (1.0 - z4) + (eF - eP) * f * z4;
      const double dx = dP + dac * f / fpp * (1.0 - z4) + (dF - dP) * f * z4;
      const double dz = ac / fpp * (df * (1.0 - z4) - 4.0 * z3 * f) + (eF - eP) * (df * z4 + 4.0 * z3 * f);
      const double base = ec - x / 6.0 * dx;
      va = base + (1.0 - z) * dz;
      vb = base - (1.0 + z) * dz;
    }
    if (czk) czk[i] = ec;
    if (cva) cva[i] = va;
    if (cvb) cvb[i] = vb;
  }
}

// 1 when any density of the current epc17-2 call is below 1e-200 (reset by
// the first kernel of each call; calls that overlap on the device race on it)
__device__ int g_epc_tiny = 0;

__global__ void epc_reset_kernel() { g_epc_tiny = 0; }

__global__ void epc_flag_kernel(long n, const double *__restrict__ rE,
                                const double *__restrict__ rN) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool tiny = i < n && (fmax(rE[i], 0.0) < 1.0e-200 || fmax(rN[i], 0.0) < 1.0e-200);
  if (__any_sync(0xffffffffu, tiny) && (threadIdx.x & 31) == 0) atomicOr(&g_epc_tiny, 1);
}

__global__ void epc17_2_kernel(long n, const double *__restrict__ rE,
                               const double *__restrict__ rN, double *__restrict__ ene,
                               double *__restrict__ pE, double *__restrict__ pN) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = 2.35, b = 2.4, c = 6.6;
  // densities below zero (rounding far from every centre) count as zero; the
  // square roots would give NaN (nAPMO's numpy restatement returns NaN there)
  const double e = fmax(rE[i], 0.0), q = fmax(rN[i], 0.0);
  const double den = a - b * sqrt(e * q) + c * e * q;
  if (ene) ene[i] = -q / den;
  double pa, pb;
  if (g_epc_tiny) {
    pa = (b * sqrt(e) * pow(q, 1.5) - 2.0 * a * q) / (den * den) / 2.0;
    pb = (b * sqrt(q) * pow(e, 1.5) - 2.0 * a * e) / (den * den) / 2.0;
  } else {
    const double s = sqrt(e * q);
    pa = (e * q * (c * q - b * q / (2.0 * s)) - q * den) / (den * den);
    pb = (q * e * (c * e - b * e / (2.0 * s)) - e * den) / (den * den);
  }
  if (pE) pE[i] = pa;
  if (pN) pN[i] = pb;
}

}  // namespace
}  // namespace napmo

using namespace napmo;

extern "C" {

// LDA exchange and VWN5 correlation of rho (device, n values): energies per
// particle and potentials (device outputs; any may be null).  Replaces
// Functional.compute_exchange / compute_correlation of nAPMO's 'lda'
// (xc_interface.py:62-90, LibXC lda_x and lda_c_vwn, unpolarised).
int napmo_gpu_lda_xc(long n, const double *rho, double *x_zk, double *x_vrho, double *c_zk,
                     double *c_vrho, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(n >= 0, "negative size");
    if (n == 0) return kOk;
    lda_xc_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        n, rho, x_zk, x_vrho, c_zk, c_vrho);
    NAPMO_TRY_CUDA(cudaGetLastError(), "lda xc");
    return kOk;
  });
}

// Spin-polarised LDA exchange and VWN5 correlation of (rho_a, rho_b) (device,
// n values each): energies per particle of the total density and the
// potentials of both spins (device outputs; any may be null).  Replaces
// Functional.compute_exchange / compute_correlation with spin 'polarized'
// (xc_interface.py:62-90, LibXC lda_x and lda_c_vwn), which nAPMO's DFT uses
// for open shells (dft_solver.py:35); nAPMO interleaves the two spins in one
// array, this takes them as two.
int napmo_gpu_lda_xc_polarized(long n, const double *rho_a, const double *rho_b, double *x_zk,
                               double *x_va, double *x_vb, double *c_zk, double *c_va,
                               double *c_vb, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(n >= 0, "negative size");
    if (n == 0) return kOk;
    lda_xc_pol_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        n, rho_a, rho_b, x_zk, x_va, x_vb, c_zk, c_va, c_vb);
    NAPMO_TRY_CUDA(cudaGetLastError(), "polarised lda xc");
    return kOk;
  });
}

// epc17-2 at n common points of the electronic and nuclear densities (device):
// energy per electron and the potentials of both species (device outputs, any
// may be null); replaces epc17_2 (interspecies_correlation.py:36-68).  Calls
// that overlap on the device share the flag of tiny densities.
int napmo_gpu_epc17_2(long n, const double *rho_e, const double *rho_n, double *ene,
                      double *pot_e, double *pot_n, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(n >= 0, "negative size");
    if (n == 0) return kOk;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = (unsigned)((n + 255) / 256);
    epc_reset_kernel<<<1, 1, 0, s>>>();
    epc_flag_kernel<<<grid, 256, 0, s>>>(n, rho_e, rho_n);
    epc17_2_kernel<<<grid, 256, 0, s>>>(n, rho_e, rho_n, ene, pot_e, pot_n);
    NAPMO_TRY_CUDA(cudaGetLastError(), "epc17-2");
    return kOk;
  });
}

}  // extern "C"
