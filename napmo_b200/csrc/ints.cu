// One-electron integrals over contracted Cartesian Gaussians on the device:
// overlap S, kinetic energy T and nuclear attraction V = -sum_C Z_C <a|1/r_C|b>
// of nAPMO's normalised contracted functions (each function of unit norm, as
// LibintInterface::compute_1body_ints returns them after its `norma` scaling,
// src/ints/libint_iface.cpp:55-190; nAPMO's own primitive overlap is
// src/ints/overlap.cpp:12-64).
//
// McMurchie-Davidson scheme (T. Helgaker, P. Jorgensen, J. Olsen, Molecular
// Electronic-Structure Theory, ch. 9.5 and 9.9): per primitive pair the
// Hermite expansion coefficients E^{ij}_t of each Cartesian direction give
//   S = K (pi/p)^(3/2) E^x_0 E^y_0 E^z_0,
//   T from the overlaps with j -> j +- 2 of each direction,
//   V = -sum_C Z_C K (2 pi/p) sum_tuv E^x_t E^y_u E^z_v R_tuv(p, P - C),
// with R_tuv the Hermite Coulomb integrals built from the Boys function.
// One thread per contracted pair (mu >= nu); both triangles written.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "capi_common.cuh"
#include "host.h"

namespace napmo {
namespace {

// Contracted functions flattened for the device: primitive k of function f
// is start[f] <= k < start[f+1]; coef = c_k x primitive norm x contraction norm.
struct FuncTable {
  int n = 0;
  const int *start = nullptr;
  const double *zeta = nullptr;
  const double *coef = nullptr;
  const int *l = nullptr;         // [n][3]
  const double *origin = nullptr; // [n][3]
};

// 1 / (2j + 1) for j < kInvOdd: the series and the downward recursion below
// multiply by these instead of dividing (one FP64 division per series term
// would dominate the kernel)
// (IEEE divisions folded at compile time; the table is part of the module
// image, so it is in place whenever the module is loaded, with no upload).
constexpr int kInvOdd = 320;
struct InvOddTable {
  double v[kInvOdd];
  constexpr InvOddTable() : v() {
    for (int j = 0; j < kInvOdd; ++j) v[j] = 1.0 / (2 * j + 1);
  }
};
__device__ const InvOddTable g_inv_odd_table;
#define g_inv_odd (g_inv_odd_table.v)

// Boys function F_m(T) for m = 0..mmax.  T < 35: the series at mmax,
//   F_m(T) = e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
// (all terms positive), then the downward recursion
//   F_m = (2T F_(m+1) + e^-T) / (2m+1);
// T >= 35: F_0 = sqrt(pi/T) erf(sqrt(T)) / 2 and the upward recursion
//   F_(m+1) = ((2m+1) F_m - e^-T) / (2T).
__device__ void boys(int mmax, double T, double *F) {
  const double e = exp(-T);
  if (T < 35.0) {
    const double t2 = 2.0 * T;
    double term = __ldg(&g_inv_odd[mmax]), sum = term;
    for (int k = 1; k < 256; ++k) {  // mmax + k < 8 + 256 <= kInvOdd
      term *= t2 * __ldg(&g_inv_odd[mmax + k]);
      sum += term;
      if (term < 1e-17 * sum) break;
    }
    F[mmax] = e * sum;
    for (int m = mmax - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * __ldg(&g_inv_odd[m]);
  } else {
    F[0] = 0.5 * sqrt(M_PI / T) * erf(sqrt(T));
    for (int m = 0; m < mmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
  }
}

// One Cartesian direction of a primitive pair: the Hermite coefficients
// E^{la,lb}_t (t <= la + lb) and the overlap-type values E^{la,j}_0 for
// j = lb - 2, lb + 2 (kinetic energy), without the exponential prefactor:
//   E^{i+1,j}_t = E^{ij}_(t-1) / (2p) + X_PA E^{ij}_t + (t+1) E^{ij}_(t+1)
//   E^{i,j+1}_t = E^{ij}_(t-1) / (2p) + X_PB E^{ij}_t + (t+1) E^{ij}_(t+1)
// (raised in i at j = 0, then in j; two rolling rows).
template <int L>
__device__ void hermite_dir(int la, int lb, double PA, double PB, double oo2p,
                            double (&Et)[2 * L + 1], double &s0, double &sp2, double &sm2) {
  constexpr int NT = 2 * L + 4;
  double cur[NT], nxt[NT];
  for (int t = 0; t < NT; ++t) cur[t] = 0.0;
  cur[0] = 1.0;
  for (int i = 0; i < la; ++i) {
    for (int t = 0; t < NT; ++t) {
      double v = PA * cur[t];
      if (t > 0) v += oo2p * cur[t - 1];
      if (t + 1 < NT) v += (t + 1) * cur[t + 1];
      nxt[t] = t <= i + 1 ? v : 0.0;
    }
    for (int t = 0; t < NT; ++t) cur[t] = nxt[t];
  }
  sm2 = 0.0;
  for (int j = 0; j <= lb + 2; ++j) {
    if (j == lb - 2) sm2 = cur[0];
    if (j == lb) {
      s0 = cur[0];
      for (int t = 0; t < 2 * L + 1; ++t) Et[t] = cur[t];
    }
    if (j == lb + 2) {
      sp2 = cur[0];
      break;
    }
    for (int t = 0; t < NT; ++t) {
      double v = PB * cur[t];
      if (t > 0) v += oo2p * cur[t - 1];
      if (t + 1 < NT) v += (t + 1) * cur[t + 1];
      nxt[t] = t <= la + j + 1 ? v : 0.0;
    }
    for (int t = 0; t < NT; ++t) cur[t] = nxt[t];
  }
}

// Largest (Lt+1)(Lx+1)(Ly+1)(Lz+1) over Lx + Ly + Lz = Lt <= 2L: 60 for d
// functions (2, 1, 1), 189 for f (2, 2, 2).
template <int L>
struct RSize {
  static constexpr int value = L <= 2 ? 64 : 192;
};

// L = largest Cartesian exponent sum of one function supported by the instance.
template <int L>
__global__ void __launch_bounds__(128)
one_body_kernel(FuncTable B, int nq, const double *__restrict__ q, double *__restrict__ S,
                double *__restrict__ T, double *__restrict__ V, long npair) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= npair) return;
  int mu = (int)((sqrt(8.0 * (double)e + 1.0) - 1.0) * 0.5);
  while ((long)mu * (mu + 1) / 2 > e) --mu;
  while ((long)(mu + 1) * (mu + 2) / 2 <= e) ++mu;
  const int nu = (int)(e - (long)mu * (mu + 1) / 2);
  int la[3], lb[3];
  double A[3], Bc[3];
  for (int d = 0; d < 3; ++d) {
    la[d] = B.l[mu * 3 + d];
    lb[d] = B.l[nu * 3 + d];
    A[d] = B.origin[mu * 3 + d];
    Bc[d] = B.origin[nu * 3 + d];
  }
  const int Lx = la[0] + lb[0], Ly = la[1] + lb[1], Lz = la[2] + lb[2];
  const int Lt = Lx + Ly + Lz;
  const int ny = Ly + 1, nz = Lz + 1, nxyz = (Lx + 1) * ny * nz;
  const bool fits = (Lt + 1) * nxyz <= RSize<L>::value;
  double s_acc = 0.0, t_acc = 0.0, v_acc = fits ? 0.0 : nan("");
  double AB2 = 0.0;
  for (int d = 0; d < 3; ++d) AB2 += (A[d] - Bc[d]) * (A[d] - Bc[d]);
  for (int kp = B.start[mu]; kp < B.start[mu + 1]; ++kp) {
    const double a = B.zeta[kp];
    for (int lp = B.start[nu]; lp < B.start[nu + 1]; ++lp) {
      const double b = B.zeta[lp];
      const double p = a + b, oo2p = 0.5 / p;
      const double cc = B.coef[kp] * B.coef[lp] * exp(-a * b / p * AB2);
      const double sq = sqrt(M_PI / p);
      double Et[3][2 * L + 1], P[3], Sd[3], Td[3];
      for (int d = 0; d < 3; ++d) {
        P[d] = (a * A[d] + b * Bc[d]) / p;
        double s0, sp2, sm2;
        hermite_dir<L>(la[d], lb[d], P[d] - A[d], P[d] - Bc[d], oo2p, Et[d], s0, sp2, sm2);
        const int j = lb[d];
        Sd[d] = sq * s0;
        Td[d] = sq * (-2.0 * b * b * sp2 + b * (2 * j + 1) * s0 - 0.5 * j * (j - 1) * sm2);
      }
      s_acc += cc * Sd[0] * Sd[1] * Sd[2];
      t_acc += cc * (Td[0] * Sd[1] * Sd[2] + Sd[0] * Td[1] * Sd[2] + Sd[0] * Sd[1] * Td[2]);
      if (!V || !fits) continue;
      double sum_c = 0.0;
      for (int c = 0; c < nq; ++c) {
        const double X = P[0] - q[c * 4 + 0], Y = P[1] - q[c * 4 + 1], Z = P[2] - q[c * 4 + 2];
        double F[2 * L + 1];
        boys(Lt, p * (X * X + Y * Y + Z * Z), F);
        // R^n_tuv at [n][t][u][v] (packed extents), in order of increasing t + u + v
        double R[RSize<L>::value];
        auto at = [&](int n, int t, int u, int v) { return ((n * (Lx + 1) + t) * ny + u) * nz + v; };
        double m2p = 1.0;
        for (int n = 0; n <= Lt; ++n) {
          R[at(n, 0, 0, 0)] = m2p * F[n];
          m2p *= -2.0 * p;
        }
        for (int sum = 1; sum <= Lt; ++sum)
          for (int t = 0; t <= min(sum, Lx); ++t)
            for (int u = 0; u <= min(sum - t, Ly); ++u) {
              const int v = sum - t - u;
              if (v > Lz) continue;
              for (int n = 0; n <= Lt - sum; ++n) {
                double r;
                if (t > 0)
                  r = X * R[at(n + 1, t - 1, u, v)] +
                      (t > 1 ? (t - 1) * R[at(n + 1, t - 2, u, v)] : 0.0);
                else if (u > 0)
                  r = Y * R[at(n + 1, t, u - 1, v)] +
                      (u > 1 ? (u - 1) * R[at(n + 1, t, u - 2, v)] : 0.0);
                else
                  r = Z * R[at(n + 1, t, u, v - 1)] +
                      (v > 1 ? (v - 1) * R[at(n + 1, t, u, v - 2)] : 0.0);
                R[at(n, t, u, v)] = r;
              }
            }
        double acc = 0.0;
        for (int t = 0; t <= Lx; ++t)
          for (int u = 0; u <= Ly; ++u)
            for (int v = 0; v <= Lz; ++v)
              acc += Et[0][t] * Et[1][u] * Et[2][v] * R[at(0, t, u, v)];
        sum_c += q[c * 4 + 3] * acc;
      }
      v_acc -= cc * (2.0 * M_PI / p) * sum_c;
    }
  }
  const long n = B.n;
  if (S) S[mu * n + nu] = S[nu * n + mu] = s_acc;
  if (T) T[mu * n + nu] = T[nu * n + mu] = t_acc;
  if (V) V[mu * n + nu] = V[nu * n + mu] = v_acc;
}

// The same integrals with one warp per contracted pair: the primitive loops
// run in step across the warp and the lanes share the point charges, then
// one shuffle reduction (the thread-per-pair kernel diverges on the
// primitive counts and angular momenta of neighbouring pairs; with many
// charges this mapping keeps the lanes busy).
template <int L>
__global__ void __launch_bounds__(128)
one_body_warp_kernel(FuncTable B, int nq, const double *__restrict__ q, double *__restrict__ S,
                     double *__restrict__ T, double *__restrict__ V, long npair) {
  const long e = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // one pair per warp
  const int lane = threadIdx.x & 31;
  if (e >= npair) return;
  int mu = (int)((sqrt(8.0 * (double)e + 1.0) - 1.0) * 0.5);
  while ((long)mu * (mu + 1) / 2 > e) --mu;
  while ((long)(mu + 1) * (mu + 2) / 2 <= e) ++mu;
  const int nu = (int)(e - (long)mu * (mu + 1) / 2);
  int la[3], lb[3];
  double A[3], Bc[3];
  for (int d = 0; d < 3; ++d) {
    la[d] = B.l[mu * 3 + d];
    lb[d] = B.l[nu * 3 + d];
    A[d] = B.origin[mu * 3 + d];
    Bc[d] = B.origin[nu * 3 + d];
  }
  const int Lx = la[0] + lb[0], Ly = la[1] + lb[1], Lz = la[2] + lb[2];
  const int Lt = Lx + Ly + Lz;
  const int ny = Ly + 1, nz = Lz + 1, nxyz = (Lx + 1) * ny * nz;
  const bool fits = (Lt + 1) * nxyz <= RSize<L>::value;
  double s_acc = 0.0, t_acc = 0.0, v_acc = fits ? 0.0 : nan("");
  double AB2 = 0.0;
  for (int d = 0; d < 3; ++d) AB2 += (A[d] - Bc[d]) * (A[d] - Bc[d]);
  for (int kp = B.start[mu]; kp < B.start[mu + 1]; ++kp) {
    const double a = B.zeta[kp];
    for (int lp = B.start[nu]; lp < B.start[nu + 1]; ++lp) {
      const double b = B.zeta[lp];
      const double p = a + b, oo2p = 0.5 / p;
      const double cc = B.coef[kp] * B.coef[lp] * exp(-a * b / p * AB2);
      const double sq = sqrt(M_PI / p);
      double Et[3][2 * L + 1], P[3], Sd[3], Td[3];
      for (int d = 0; d < 3; ++d) {
        P[d] = (a * A[d] + b * Bc[d]) / p;
        double s0, sp2, sm2;
        hermite_dir<L>(la[d], lb[d], P[d] - A[d], P[d] - Bc[d], oo2p, Et[d], s0, sp2, sm2);
        const int j = lb[d];
        Sd[d] = sq * s0;
        Td[d] = sq * (-2.0 * b * b * sp2 + b * (2 * j + 1) * s0 - 0.5 * j * (j - 1) * sm2);
      }
      s_acc += cc * Sd[0] * Sd[1] * Sd[2];
      t_acc += cc * (Td[0] * Sd[1] * Sd[2] + Sd[0] * Td[1] * Sd[2] + Sd[0] * Sd[1] * Td[2]);
      if (!V || !fits) continue;
      double sum_c = 0.0;
      for (int c = lane; c < nq; c += 32) {
        const double X = P[0] - q[c * 4 + 0], Y = P[1] - q[c * 4 + 1], Z = P[2] - q[c * 4 + 2];
        double F[2 * L + 1];
        boys(Lt, p * (X * X + Y * Y + Z * Z), F);
        double R[RSize<L>::value];
        auto at = [&](int n, int t, int u, int v) { return ((n * (Lx + 1) + t) * ny + u) * nz + v; };
        double m2p = 1.0;
        for (int n = 0; n <= Lt; ++n) {
          R[at(n, 0, 0, 0)] = m2p * F[n];
          m2p *= -2.0 * p;
        }
        for (int sum = 1; sum <= Lt; ++sum)
          for (int t = 0; t <= min(sum, Lx); ++t)
            for (int u = 0; u <= min(sum - t, Ly); ++u) {
              const int v = sum - t - u;
              if (v > Lz) continue;
              for (int n = 0; n <= Lt - sum; ++n) {
                double r;
                if (t > 0)
                  r = X * R[at(n + 1, t - 1, u, v)] +
                      (t > 1 ? (t - 1) * R[at(n + 1, t - 2, u, v)] : 0.0);
                else if (u > 0)
                  r = Y * R[at(n + 1, t, u - 1, v)] +
                      (u > 1 ? (u - 1) * R[at(n + 1, t, u - 2, v)] : 0.0);
                else
                  r = Z * R[at(n + 1, t, u, v - 1)] +
                      (v > 1 ? (v - 1) * R[at(n + 1, t, u, v - 2)] : 0.0);
                R[at(n, t, u, v)] = r;
              }
            }
        double acc = 0.0;
        for (int t = 0; t <= Lx; ++t)
          for (int u = 0; u <= Ly; ++u)
            for (int v = 0; v <= Lz; ++v)
              acc += Et[0][t] * Et[1][u] * Et[2][v] * R[at(0, t, u, v)];
        sum_c += q[c * 4 + 3] * acc;
      }
      v_acc -= cc * (2.0 * M_PI / p) * sum_c;
    }
  }
  for (int o = 16; o > 0; o >>= 1) v_acc += __shfl_down_sync(0xffffffffu, v_acc, o);
  if (lane != 0) return;
  const long n = B.n;
  if (S) S[mu * n + nu] = S[nu * n + mu] = s_acc;
  if (T) T[mu * n + nu] = T[nu * n + mu] = t_acc;
  if (V) V[mu * n + nu] = V[nu * n + mu] = v_acc;
}

// Point charges from which the warp-per-pair kernel is used.
constexpr int kWarpCharges = 16;

// Host image of a FuncTable.
struct HostFuncs {
  std::vector<int> start{0}, l;
  std::vector<double> zeta, coef, origin;
  int max_l = 0;
  void add(const ContractedGaussian &c) {
    for (const auto &p : c.prim) {
      zeta.push_back(p.zeta);
      coef.push_back(p.coeff * p.norma * c.norma);
    }
    start.push_back((int)zeta.size());
    int L = 0;
    for (int d = 0; d < 3; ++d) {
      l.push_back(c.l[d]);
      origin.push_back(c.origin[d]);
      L += c.l[d];
    }
    max_l = std::max(max_l, L);
  }
  int n() const { return (int)start.size() - 1; }
};

// S, T, V (device [n][n], any null) of the functions in h and the charges
// (host [nq][4]: x, y, z, Z); scratch from the stream-ordered allocator.
int one_body_device(const HostFuncs &h, int nq, const double *charges, double *S, double *T,
                    double *V, cudaStream_t s) {
  const int n = h.n();
  if (n == 0) return kOk;
  if (h.max_l > 3)
    return set_error(kNotSupported, "one-electron integrals support functions up to f");
  const size_t np = h.zeta.size();
  const size_t bytes = (h.start.size() + h.l.size()) * sizeof(int) +
                       (2 * np + h.origin.size() + 4 * (size_t)nq) * sizeof(double) + 64;
  char *ws = nullptr;
  NAPMO_TRY_CUDA(cudaMallocAsync((void **)&ws, bytes, s), "one-body workspace");
  double *dz = (double *)ws, *dc = dz + np, *dor = dc + np, *dq = dor + h.origin.size();
  int *dstart = (int *)(dq + 4 * (size_t)nq), *dl = dstart + h.start.size();
  cudaError_t e = cudaMemcpyAsync(dz, h.zeta.data(), np * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dc, h.coef.data(), np * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dor, h.origin.data(), h.origin.size() * sizeof(double),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nq > 0)
    e = cudaMemcpyAsync(dq, charges, 4 * (size_t)nq * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dstart, h.start.data(), h.start.size() * sizeof(int),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dl, h.l.data(), h.l.size() * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    FuncTable B;
    B.n = n;
    B.start = dstart;
    B.zeta = dz;
    B.coef = dc;
    B.l = dl;
    B.origin = dor;
    const long npair = (long)n * (n + 1) / 2;
    if (V && nq >= kWarpCharges) {  // many charges: one warp per pair
      const unsigned grid = (unsigned)((npair + 3) / 4);
      if (h.max_l <= 2)
        one_body_warp_kernel<2><<<grid, 128, 0, s>>>(B, nq, dq, S, T, V, npair);
      else
        one_body_warp_kernel<3><<<grid, 128, 0, s>>>(B, nq, dq, S, T, V, npair);
    } else {
      const unsigned grid = (unsigned)((npair + 127) / 128);
      if (h.max_l <= 2)
        one_body_kernel<2><<<grid, 128, 0, s>>>(B, nq, dq, S, T, V, npair);
      else
        one_body_kernel<3><<<grid, 128, 0, s>>>(B, nq, dq, S, T, V, npair);
    }
    e = cudaGetLastError();
  }
  // the host images must outlive the copies
  const cudaError_t es = cudaStreamSynchronize(s);
  cudaFreeAsync(ws, s);
  NAPMO_TRY_CUDA(e, "one-body integrals");
  NAPMO_TRY_CUDA(es, "one-body integrals");
  return kOk;
}

}  // namespace

// nAPMO's LibintInterface for the one-body part: the bases of one species and
// the point charges (libint_iface.cpp:41-134).
struct OneBodyInterface {
  std::vector<BasisSet *> bases;
  std::vector<double> charges;  // [nq][4]
  int nbasis = 0;
};

}  // namespace napmo

using namespace napmo;

extern "C" {

// S, T and V = -sum_C Z_C <mu|1/r_C|nu> of basis b (device outputs [n][n],
// any may be null; charges host [nq][4] = x, y, z, Z in bohr).  Replaces
// libint's one-body engines behind LibintInterface_compute_1body_ints
// (libint_iface.cpp:136-190) and the primitive overlap of overlap.cpp:12-64.
int napmo_gpu_one_body(BasisSet *b, int nq, const double *charges, double *S, double *T,
                       double *V, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(nq >= 0 && (nq == 0 || charges), "charges missing");
    HostFuncs h;
    for (const auto &c : b->cont) h.add(c);
    return one_body_device(h, nq, charges, S, T, V, (cudaStream_t)stream);
  });
}

void *LibintInterface_new(int) {
  void *out = nullptr;
  guarded([&] {
    out = new OneBodyInterface;
    return kOk;
  });
  return out;
}

void LibintInterface_del(void *l) { delete (OneBodyInterface *)l; }

void LibintInterface_add_basis(void *l, void *b) {
  guarded([&] {
    auto *L = (OneBodyInterface *)l;
    NAPMO_REQUIRE(L && b, "null interface or basis");
    L->bases.push_back((BasisSet *)b);
    L->nbasis += (int)((BasisSet *)b)->cont.size();
    return kOk;
  });
}

void LibintInterface_add_pointcharges(void *l, int z, double *center) {
  guarded([&] {
    auto *L = (OneBodyInterface *)l;
    NAPMO_REQUIRE(L && center, "null interface or centre");
    L->charges.insert(L->charges.end(), {center[0], center[1], center[2], (double)z});
    return kOk;
  });
}

int LibintInterface_get_nbasis(void *l) { return l ? ((OneBodyInterface *)l)->nbasis : 0; }

// kind 1 overlap, 2 kinetic, 3 nuclear attraction (host result [n][n]),
// libint_iface.cpp:1318-1345.
void LibintInterface_compute_1body_ints(void *l, int kind, double *result) {
  guarded([&] {
    auto *L = (OneBodyInterface *)l;
    NAPMO_REQUIRE(L && result, "null interface or result");
    NAPMO_REQUIRE(kind >= 1 && kind <= 3, "integral kind must be 1, 2 or 3");
    HostFuncs h;
    for (auto *b : L->bases)
      for (const auto &c : b->cont) h.add(c);
    const int n = h.n();
    if (n == 0) return kOk;
    cudaStream_t s = host_api_stream();
    DevBuf<double> out;
    NAPMO_TRY_CUDA(out.alloc((size_t)n * n), "alloc");
    const int nq = (int)L->charges.size() / 4;
    int st = one_body_device(h, nq, L->charges.data(), kind == 1 ? out.p : nullptr,
                             kind == 2 ? out.p : nullptr, kind == 3 ? out.p : nullptr, s);
    if (st) return st;
    NAPMO_TRY_CUDA(cudaMemcpyAsync(result, out.p, (size_t)n * n * sizeof(double),
                                   cudaMemcpyDeviceToHost, s),
                   "download");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "sync");
    return kOk;
  });
}

}  // extern "C"
