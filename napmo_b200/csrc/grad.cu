// Nuclear-coordinate gradient of the grid quadrature energy of one species in
// an external point-charge potential:
//
//   E(D, R) = sum_p wq_p wb_p(R) rho_D(r_p; R) v(r_p; R),
//   rho_D(r) = sum_{mu,nu} D[mu][nu] phi_mu(r) phi_nu(r),
//   v(r)     = sum_C q_C / |r - R_C|,
//
// where every grid point moves with its atom (r_p = R_A(p) + r_i u_j,
// atomic_grid.cpp:12-51), wb are Becke's cell weights (becke.cpp:79-176),
// phi_mu is centred on an atom (gto.cpp:41-51) and each charge sits at a
// given position.  dE/dD is the quadrature matrix of wq wb v
// (nwavefunction.cpp:161-197); this file gives dE/dR_B for the grid centres,
// the sum of
//
//   Becke:    wq rho v d wb / dR_B           (cell functions of all pairs,
//                                             distances to the point and R_KL)
//   basis:    2 W v sum_mu T_mu grad phi_mu  (T = D phi) with + for B = A(p)
//             (point motion) and - for B = centre of mu
//   charges:  W rho grad_r v for B = A(p)
//
// and dE/dR_C = sum_p W rho q_C (r_p - R_C)/|r_p - R_C|^3 for each charge
// (the caller adds it to the atom that carries the charge, if any)
//
// with W = wq wb.  One thread per point recomputes phi and grad phi (two
// passes over the shells) instead of storing them; per-thread contributions
// are reduced per CTA (warp shuffles, then warps in order) into
// partial[block][3 nc + 3 nq + 1] and summed over blocks in a fixed order.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "capi_common.cuh"
#include "host.h"
#include "kernels.cuh"

namespace napmo {

int basis_device(BasisSet *b, cudaStream_t s, const DeviceBasis **out);

namespace {

constexpr int kGradThreads = 128;
constexpr int kMaxGradAtoms = 16;
constexpr int kMaxGradCharges = 16;
constexpr int kMaxGradBasis = 192;
constexpr int kMaxComp = 15;

struct GradArgs {
  int npoint, nc, n, nq;
  const double *x, *y, *z, *wq, *wb;
  const double *origin;  // [nc][3]
  const double *Rt, *at; // packed lower triangles R_ij, a_ij (becke.cpp:80-115)
  const int *off;        // [nc + 1] point offsets of the atoms
  DeviceBasis basis;
  const int *shell_atom; // atom of each shell
  const double *D;       // [n][n]
  const double *q;       // [nq][4]: x, y, z, charge
  double *partial;       // [gridDim][3 nc + 3 nq + 1]
};

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

// s(nu) = (1 - f(f(f(nu)))) / 2, f(x) = x (3 - x^2) / 2, and ds/dnu.
__device__ __forceinline__ void cell(double nu, double &s, double &ds) {
  double x = nu, d = 1.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    d *= 1.5 * (1.0 - x * x);
    x = 0.5 * x * (3.0 - x * x);
  }
  s = 0.5 * (1.0 - x);
  ds = -0.5 * d;
}

__global__ void __launch_bounds__(kGradThreads) grad_kernel(GradArgs g) {
  extern __shared__ double red[];  // [warps][ncomp]
  const int nc = g.nc, nq3 = 3 * g.nq, ncomp = 3 * nc + nq3 + 1;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[3 * kMaxGradAtoms + 3 * kMaxGradCharges + 1];
  for (int i = 0; i < ncomp; ++i) acc[i] = 0.0;

  if (p < g.npoint) {
    const double px = g.x[p], py = g.y[p], pz = g.z[p];
    int A = 0;
    while (A + 1 < nc && g.off[A + 1] <= p) ++A;
    // ---- basis values and T = D phi
    double phi[kMaxGradBasis], T[kMaxGradBasis];
    const DeviceBasis &b = g.basis;
    for (int s = 0; s < b.nshell; ++s) {
      const int *info = b.shell_info + 6 * s;
      const int f0 = info[0], ncomp_s = info[1], p0 = info[2], np = info[3], c0 = info[4];
      const double *cen = b.shell_center + 4 * s;
      const double dx = px - cen[0], dy = py - cen[1], dz = pz - cen[2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      double e[kMaxComp];
      for (int c = 0; c < ncomp_s; ++c) e[c] = 0.0;
      if (cen[3] * r2 <= 746.0)
        for (int k = 0; k < np; ++k) {
          const double ex = exp(-b.prim_zeta[p0 + k] * r2);
          for (int c = 0; c < ncomp_s; ++c) e[c] += b.coef[c0 + c * np + k] * ex;
        }
      for (int c = 0; c < ncomp_s; ++c) {
        const int f = f0 + c;
        phi[f] = ipow(dx, b.func_l[3 * f]) * ipow(dy, b.func_l[3 * f + 1]) *
                 ipow(dz, b.func_l[3 * f + 2]) * e[c];
      }
    }
    double rho = 0.0;
    for (int mu = 0; mu < g.n; ++mu) {
      double t = 0.0;
      const double *Drow = g.D + (long)mu * g.n;
      for (int nu = 0; nu < g.n; ++nu) t = fma(Drow[nu], phi[nu], t);
      T[mu] = t;
      rho = fma(phi[mu], t, rho);
    }
    // ---- potential and its gradient at the point
    double v = 0.0, gvx = 0.0, gvy = 0.0, gvz = 0.0;
    for (int c = 0; c < g.nq; ++c) {
      const double *qc = g.q + 4 * c;
      const double dx = px - qc[0], dy = py - qc[1], dz = pz - qc[2];
      const double d2 = dx * dx + dy * dy + dz * dz, id = 1.0 / sqrt(d2);
      const double t = qc[3] * id * id * id;
      v += qc[3] * id;
      gvx -= t * dx;
      gvy -= t * dy;
      gvz -= t * dz;
      acc[3 * nc + 3 * c] = t * dx;  // moving the charge; scaled by W rho below
      acc[3 * nc + 3 * c + 1] = t * dy;
      acc[3 * nc + 3 * c + 2] = t * dz;
    }
    const double W = g.wq[p] * g.wb[p];
    for (int i = 0; i < nq3; ++i) acc[3 * nc + i] *= W * rho;
    acc[3 * A] += W * rho * gvx;
    acc[3 * A + 1] += W * rho * gvy;
    acc[3 * A + 2] += W * rho * gvz;
    acc[3 * nc + nq3] = W * rho * v;  // energy
    // ---- basis gradients: 2 W v T_mu grad phi_mu
    const double cb = 2.0 * W * v;
    for (int s = 0; s < b.nshell; ++s) {
      const int *info = b.shell_info + 6 * s;
      const int f0 = info[0], ncomp_s = info[1], p0 = info[2], np = info[3], c0 = info[4];
      const double *cen = b.shell_center + 4 * s;
      const double dx = px - cen[0], dy = py - cen[1], dz = pz - cen[2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (cen[3] * r2 > 746.0) continue;
      double e[kMaxComp], ez[kMaxComp];
      for (int c = 0; c < ncomp_s; ++c) e[c] = ez[c] = 0.0;
      for (int k = 0; k < np; ++k) {
        const double zeta = b.prim_zeta[p0 + k];
        const double ex = exp(-zeta * r2);
        for (int c = 0; c < ncomp_s; ++c) {
          const double t = b.coef[c0 + c * np + k] * ex;
          e[c] += t;
          ez[c] += t * zeta;
        }
      }
      double hx = 0.0, hy = 0.0, hz = 0.0;
      for (int c = 0; c < ncomp_s; ++c) {
        const int f = f0 + c;
        const int lx = b.func_l[3 * f], ly = b.func_l[3 * f + 1], lz = b.func_l[3 * f + 2];
        const double px_ = ipow(dx, lx), py_ = ipow(dy, ly), pz_ = ipow(dz, lz);
        const double gx = (lx ? lx * ipow(dx, lx - 1) * e[c] : 0.0) - 2.0 * ipow(dx, lx + 1) * ez[c];
        const double gy = (ly ? ly * ipow(dy, ly - 1) * e[c] : 0.0) - 2.0 * ipow(dy, ly + 1) * ez[c];
        const double gz = (lz ? lz * ipow(dz, lz - 1) * e[c] : 0.0) - 2.0 * ipow(dz, lz + 1) * ez[c];
        const double t = cb * T[f];
        hx += t * gx * py_ * pz_;
        hy += t * px_ * gy * pz_;
        hz += t * px_ * py_ * gz;
      }
      const int a = g.shell_atom[s];
      acc[3 * A] += hx;
      acc[3 * A + 1] += hy;
      acc[3 * A + 2] += hz;
      acc[3 * a] -= hx;
      acc[3 * a + 1] -= hy;
      acc[3 * a + 2] -= hz;
    }
    // ---- Becke weights: d wb / dR_B, coefficient wq rho v
    {
      double rK[kMaxGradAtoms], uK[kMaxGradAtoms][3];
      for (int k = 0; k < nc; ++k) {
        const double dx = px - g.origin[3 * k], dy = py - g.origin[3 * k + 1],
                     dz = pz - g.origin[3 * k + 2];
        rK[k] = sqrt(dx * dx + dy * dy + dz * dz);
        const double ir = rK[k] > 0.0 ? 1.0 / rK[k] : 0.0;
        uK[k][0] = dx * ir;
        uK[k][1] = dy * ir;
        uK[k][2] = dz * ir;
      }
      double P[kMaxGradAtoms];
      double Z = 0.0;
      for (int k = 0; k < nc; ++k) {
        double prod = 1.0;
        for (int l = 0; l < nc; ++l) {
          if (l == k) continue;
          const int o = (k < l) ? l * (l + 1) / 2 + k : k * (k + 1) / 2 + l;
          const double mu = (rK[k] - rK[l]) / g.Rt[o];
          const double as = (k < l ? -1.0 : 1.0) * g.at[o];
          double s, ds;
          cell(mu + as * (1.0 - mu * mu), s, ds);
          prod *= s;
        }
        P[k] = prod;
        Z += prod;
      }
      const double w = P[A] / Z;
      const double cw = g.wq[p] * rho * v / Z;
      double gr[3] = {0.0, 0.0, 0.0};  // through the point (moves with A)
      for (int k = 0; k < nc; ++k) {
        const double alpha = cw * ((k == A ? 1.0 : 0.0) - w);
        if (alpha == 0.0) continue;
        for (int l = 0; l < nc; ++l) {
          if (l == k) continue;
          // product of the other cell functions of k (recomputed: no division by s)
          double excl = 1.0, ds_kl = 0.0, mu_kl = 0.0, R = 0.0;
          for (int m = 0; m < nc; ++m) {
            if (m == k) continue;
            const int o = (k < m) ? m * (m + 1) / 2 + k : k * (k + 1) / 2 + m;
            const double mu = (rK[k] - rK[m]) / g.Rt[o];
            const double as = (k < m ? -1.0 : 1.0) * g.at[o];
            double s, ds;
            cell(mu + as * (1.0 - mu * mu), s, ds);
            if (m == l) {
              ds_kl = ds * (1.0 - 2.0 * as * mu);
              mu_kl = mu;
              R = g.Rt[o];
            } else {
              excl *= s;
            }
          }
          const double t = alpha * excl * ds_kl / R;
          double e_kl[3];
          for (int d = 0; d < 3; ++d) e_kl[d] = (g.origin[3 * k + d] - g.origin[3 * l + d]) / R;
          for (int d = 0; d < 3; ++d) {
            gr[d] += t * (uK[k][d] - uK[l][d]);
            acc[3 * k + d] += t * (-uK[k][d] - mu_kl * e_kl[d]);
            acc[3 * l + d] += t * (uK[l][d] + mu_kl * e_kl[d]);
          }
        }
      }
      for (int d = 0; d < 3; ++d) acc[3 * A + d] += gr[d];
    }
  }
  // ---- deterministic CTA reduction
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int i = 0; i < ncomp; ++i) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp * ncomp + i] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < ncomp; i += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < nw; ++w) v += red[w * ncomp + i];
    g.partial[(long)blockIdx.x * ncomp + i] = v;
  }
}

__global__ void grad_reduce_kernel(int nblock, int ncomp, const double *__restrict__ partial,
                                   double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncomp) return;
  double v = 0.0;
  for (int b = 0; b < nblock; ++b) v += partial[(long)b * ncomp + i];
  out[i] = v;
}

}  // namespace
}  // namespace napmo

using namespace napmo;

extern "C" {

// E and its derivatives (host out: E, grad[ncenter][3] for the grid centres,
// grad_q[nq][3] for the charges) of the grid quadrature energy
// sum_p wq wb rho_D v of one species (basis, device D [n][n]) in the
// potential of nq point charges (host [nq][4] = x, y, z, q).  Grid points
// and basis shells move with the grid centres (every shell must sit on one).
// No counterpart in nAPMO.
int napmo_grid_energy_gradient(BeckeGrid *grid, BasisSet *basis, const double *D, int nq,
                               const double *charges, double *E, double *grad, double *grad_q,
                               void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    const int nc = grid->ncenter, n = (int)basis->cont.size();
    NAPMO_REQUIRE(nc >= 1 && nc <= kMaxGradAtoms, "gradient: 1..16 grid centres");
    NAPMO_REQUIRE(nq >= 0 && nq <= kMaxGradCharges, "gradient: 0..16 point charges");
    NAPMO_REQUIRE(n <= kMaxGradBasis, "gradient: at most 192 basis functions");
    NAPMO_REQUIRE(!grid->layout.empty(), "gradient needs a grid built from atoms");
    HostBasisPack pk;
    pack_basis(basis->cont, &pk);
    std::vector<int> shell_atom(pk.nshell, -1);
    for (int sh = 0; sh < pk.nshell; ++sh) {
      for (int a = 0; a < nc; ++a) {
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k) {
          const double t = pk.shell_center[4 * sh + k] - grid->origin[3 * a + k];
          d2 += t * t;
        }
        if (d2 < 1e-20) {
          shell_atom[sh] = a;
          break;
        }
      }
      NAPMO_REQUIRE(shell_atom[sh] >= 0, "gradient: a basis shell is not on a grid centre");
    }
    const DeviceBasis *db = nullptr;
    int e = basis_device(basis, s, &db);
    if (e) return e;
    // Becke tables: packed R_ij and clamped a_ij (becke.cpp:80-115)
    const int tri = nc * (nc + 1) / 2;
    std::vector<double> R(tri), Aa(tri);
    int o = 0;
    for (int i = 0; i < nc; ++i)
      for (int j = 0; j <= i; ++j) {
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k) {
          const double t = grid->origin[3 * i + k] - grid->origin[3 * j + k];
          d2 += t * t;
        }
        R[o] = std::sqrt(d2);
        double aux = (grid->radii[i] - grid->radii[j]) / (grid->radii[i] + grid->radii[j]);
        aux = aux / (aux * aux - 1.0);
        Aa[o] = aux > 0.45 ? 0.45 : (aux < -0.45 ? -0.45 : aux);
        ++o;
      }
    DevBuf<double> dR, dA, dq, partial, out;
    DevBuf<int> dsa;
    NAPMO_TRY_CUDA(dR.upload(R, s), "upload");
    NAPMO_TRY_CUDA(dA.upload(Aa, s), "upload");
    NAPMO_TRY_CUDA(dsa.upload(shell_atom, s), "upload");
    std::vector<double> qv(charges, charges + 4 * (size_t)nq);
    if (nq == 0) qv.assign(4, 0.0);
    NAPMO_TRY_CUDA(dq.upload(qv, s), "upload");
    const int ncomp = 3 * nc + 3 * nq + 1;
    const int nblock = (grid->size + kGradThreads - 1) / kGradThreads;
    NAPMO_TRY_CUDA(partial.alloc((size_t)nblock * ncomp), "alloc");
    NAPMO_TRY_CUDA(out.alloc(ncomp), "alloc");
    GradArgs a{grid->size, nc, n, nq, grid->dev.x, grid->dev.y, grid->dev.z, grid->dev.w,
               grid->dev.wb, grid->dev.origin, dR.p, dA.p, grid->dev.atom_offset, *db,
               dsa.p, D, dq.p, partial.p};
    const size_t smem = (size_t)(kGradThreads / 32) * ncomp * sizeof(double);
    grad_kernel<<<nblock, kGradThreads, smem, s>>>(a);
    NAPMO_TRY_CUDA(cudaGetLastError(), "gradient kernel");
    grad_reduce_kernel<<<(ncomp + 63) / 64, 64, 0, s>>>(nblock, ncomp, partial.p, out.p);
    NAPMO_TRY_CUDA(cudaGetLastError(), "gradient reduce");
    std::vector<double> h(ncomp);
    NAPMO_TRY_CUDA(cudaMemcpyAsync(h.data(), out.p, ncomp * sizeof(double),
                                   cudaMemcpyDeviceToHost, s),
                   "download");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "gradient");
    for (int i = 0; i < 3 * nc; ++i) grad[i] = h[i];
    for (int i = 0; i < 3 * nq; ++i) grad_q[i] = h[3 * nc + i];
    *E = h[3 * nc + 3 * nq];
    return kOk;
  });
}

}  // extern "C"
