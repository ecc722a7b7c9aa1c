// Contracted Cartesian Gaussian basis functions (and their gradients) on grid
// points: phi_mu(r) = N_c sum_k c_k N_k (x-Ax)^lx (y-Ay)^ly (z-Az)^lz
// exp(-zeta_k |r-A|^2), nAPMO src/system/gto.cpp:41-51,182-192.
//
// One thread per point walks the shells; the exponentials of a shell are
// evaluated once and shared by its Cartesian components.  Shells whose
// smallest exponent gives zeta_min r^2 > 746 are skipped: exp() of any
// argument below -745.2 is exactly zero in double precision, so the skip does
// not change a single value.  Output is basis-major phi[mu * ld + p] so that
// consecutive threads write consecutive addresses.
#include "common.h"
#include "kernels.cuh"

namespace napmo {

namespace {

constexpr int kGtoThreads = 128;
constexpr int kMaxComp = 15;  // Cartesian components up to L = 4

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

template <bool kGrad>
__global__ void __launch_bounds__(kGtoThreads)
gto_kernel(DeviceBasis b, int npoint, const double *__restrict__ gx,
           const double *__restrict__ gy, const double *__restrict__ gz,
           double *__restrict__ phi, long ld, double *__restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  const double px = gx[p], py = gy[p], pz = gz[p];
  const long plane = (long)b.nfunc * ld;
  for (int s = 0; s < b.nshell; ++s) {
    const int *info = b.shell_info + 6 * s;
    const int f0 = __ldg(info + 0), ncomp = __ldg(info + 1), p0 = __ldg(info + 2),
              np = __ldg(info + 3), c0 = __ldg(info + 4);
    const double *cen = b.shell_center + 4 * s;
    const double dx = px - __ldg(cen + 0);
    const double dy = py - __ldg(cen + 1);
    const double dz = pz - __ldg(cen + 2);
    double r2 = 0.0;
    r2 += dx * dx;
    r2 += dy * dy;
    r2 += dz * dz;
    double acc[kMaxComp], accz[kMaxComp];
#pragma unroll
    for (int c = 0; c < kMaxComp; ++c) {
      acc[c] = 0.0;
      accz[c] = 0.0;
    }
    if (__ldg(cen + 3) * r2 <= 746.0) {
      for (int k = 0; k < np; ++k) {
        const double zeta = __ldg(b.prim_zeta + p0 + k);
        const double e = exp(-zeta * r2);
#pragma unroll
        for (int c = 0; c < kMaxComp; ++c) {
          if (c < ncomp) {
            const double t = __ldg(b.coef + c0 + c * np + k) * e;
            acc[c] += t;
            if (kGrad) accz[c] += t * zeta;
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < kMaxComp; ++c) {
      if (c < ncomp) {
        const int f = f0 + c;
        const int lx = __ldg(b.func_l + 3 * f), ly = __ldg(b.func_l + 3 * f + 1),
                  lz = __ldg(b.func_l + 3 * f + 2);
        const double px_ = ipow(dx, lx), py_ = ipow(dy, ly), pz_ = ipow(dz, lz);
        phi[(long)f * ld + p] = px_ * py_ * pz_ * acc[c];
        if (kGrad) {
          // d/dx [x^lx e^{-zeta r^2}] = lx x^(lx-1) - 2 zeta x^(lx+1)
          const double gxv = (lx ? lx * ipow(dx, lx - 1) * acc[c] : 0.0) -
                             2.0 * ipow(dx, lx + 1) * accz[c];
          const double gyv = (ly ? ly * ipow(dy, ly - 1) * acc[c] : 0.0) -
                             2.0 * ipow(dy, ly + 1) * accz[c];
          const double gzv = (lz ? lz * ipow(dz, lz - 1) * acc[c] : 0.0) -
                             2.0 * ipow(dz, lz + 1) * accz[c];
          grad[(long)f * ld + p] = gxv * py_ * pz_;
          grad[plane + (long)f * ld + p] = px_ * gyv * pz_;
          grad[2 * plane + (long)f * ld + p] = px_ * py_ * gzv;
        }
      }
    }
  }
}

}  // namespace

cudaError_t launch_basis_values(const DeviceBasis &b, int npoint, const double *x,
                                const double *y, const double *z, double *phi,
                                long ld, double *grad, cudaStream_t s) {
  if (npoint <= 0 || b.nfunc == 0) return cudaSuccess;
  const int blocks = (npoint + kGtoThreads - 1) / kGtoThreads;
  if (grad)
    gto_kernel<true><<<blocks, kGtoThreads, 0, s>>>(b, npoint, x, y, z, phi, ld, grad);
  else
    gto_kernel<false><<<blocks, kGtoThreads, 0, s>>>(b, npoint, x, y, z, phi, ld, nullptr);
  return cudaGetLastError();
}

}  // namespace napmo
