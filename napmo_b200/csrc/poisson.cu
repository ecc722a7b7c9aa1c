// Becke-Dickson Poisson pipeline on the device (see poisson.cuh).
//
// 1. project:  f_lm(r_i) = sqrt(4 pi (2l+1)) sum_j rho wb w S_lm(u_j) / sum_j w
//    per atom and radial shell, as a small FP64 product (DMMA tiles) of the
//    shell's weighted density with the per-rule table S_lm(u_j) (reference:
//    AtomicGrid::spherical_expansion, src/grid/atomic_grid.cpp:82-136).
// 2. radial:   the Hermite FEM matrix of u'' + b u' + a u = f on the uniform
//    t-axis depends on (atom, l) only: it is assembled and factored by banded
//    LU with partial pivoting once per grid (radial_factor_kernel).  Per solve,
//    one thread per (l, m) column builds the cubic spline of f_lm, the
//    transformed FEM right-hand side and Dirichlet values, and substitutes
//    (radial_kernel; reference: poisson_solver.py:42-118, ode2.py,
//    src/horton/ode2.cpp:232-321; the reference solves each (l, m) with
//    scipy's sparse LU).  The solution splines are written as scaled cubic
//    coefficients for step 3 and as raw (y, dy/dt) for the Python API.
// 3. evaluate: v(p) = sum_A sum_lm s_lm(|p - A|) sqrt(2l+1)/sqrt(4 pi)
//    S_lm(p - A) / |p - A|^l for every point and every atom (the potential
//    extrapolation has a tail, so no cutoff applies; reference:
//    eval_decomposition_grid, src/horton/evaluate.cpp:129-220).  Templated on
//    lmax so the solid-harmonic recursion lives in registers.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.h"
#include "dmma.cuh"
#include "host.h"
#include "poisson.cuh"
#include "solid_harmonics.h"

namespace napmo {

namespace {

__constant__ double c_ov2[5 * 2 * 5 * 2];
__constant__ double c_ov3[5 * 2 * 5 * 2 * 5 * 2];
__constant__ double c_shnorm[(kMaxLmax + 1) * (kMaxLmax + 1)];  // [l][m]
// Normalised solid harmonics by a recursion along l at fixed m (evaluation
// kernel).  With q_l = a_lm z q_(l-1) - b_lm q_(l-2) and q_m = start_m, the
// rescaled q~_l = q_l / gamma_lm (gamma_m = gamma_(m+1) = 1, gamma_l =
// b_lm gamma_(l-2)) obey q~_l = A_lm z q~_(l-1) - q~_(l-2) with
// A_lm = a_lm gamma_(l-1) / gamma_l: one product and one FMA per step.  The
// coefficients multiplying q_l are scaled by gamma_lm when staged.
__constant__ double c_rec_a[(kMaxLmax + 1) * (kMaxLmax + 1)];      // A_lm at [l][m]
__constant__ double c_rec_gamma[(kMaxLmax + 1) * (kMaxLmax + 1)];  // gamma at [lm]
__constant__ double c_rec_start[kMaxLmax + 1];
// global copy of c_rec_gamma for staging loops whose lanes read different
// entries (constant memory serves one address at a time)
__device__ double g_rec_gamma[(kMaxLmax + 1) * (kMaxLmax + 1)];
// Finite-difference weights of the radial second derivative (integers over
// common denominators, host deriv2_stencils()): [0, 28) first derivative at
// the four edge nodes (7 weights each), [28, 56) second derivative, [56, 65)
// and [65, 74) the centred 9-point first and second derivative, [74, 78) the
// denominators (edge first, edge second, centred first, centred second).
__constant__ double c_fd[78];

constexpr double kPI4 = 4.0 * M_PI;
constexpr double kInvSqrt4Pi = 0.28209479177387814347;

__device__ __forceinline__ int piece_d(long c, long k, long g) {
  if (c == g) return (int)k;
  if (c == g + 1) return (int)(2 + k);
  return 4;
}

// The Hermite tables are read through a pointer: constant memory (c_ov2,
// c_ov3) where every lane of a warp reads the same entry, a shared-memory copy
// where lanes read different entries (the FEM assembly; constant memory
// would serve those one address at a time).
__device__ double ov2_d(long xmax, long i0, int d0, long i1, int d1, const double *ov2 = c_ov2) {
  const long c0 = i0 / 2, k0 = i0 % 2, c1 = i1 / 2, k1 = i1 % 2;
  if (labs(c1 - c0) >= 2) return 0.0;
  double r = 0.0;
  if (c0 >= 1 && c0 <= xmax)
    r += ov2[((piece_d(c0, k0, c0 - 1) * 2 + d0) * 5 + piece_d(c1, k1, c0 - 1)) * 2 + d1];
  if (c0 >= 0 && c0 <= xmax - 1)
    r += ov2[((piece_d(c0, k0, c0) * 2 + d0) * 5 + piece_d(c1, k1, c0)) * 2 + d1];
  return r;
}

__device__ double ov3_d(long xmax, long i0, int d0, long i1, int d1, long i2, int d2,
                       const double *ov3 = c_ov3) {
  const long c0 = i0 / 2, k0 = i0 % 2, c1 = i1 / 2, k1 = i1 % 2, c2 = i2 / 2,
             k2 = i2 % 2;
  if (labs(c1 - c0) >= 2 || labs(c2 - c0) >= 2) return 0.0;
  double r = 0.0;
  if (c0 >= 1 && c0 <= xmax) {
    const long g = c0 - 1;
    r += ov3[((((piece_d(c0, k0, g) * 2 + d0) * 5 + piece_d(c1, k1, g)) * 2 + d1) * 5 +
                piece_d(c2, k2, g)) * 2 + d2];
  }
  if (c0 >= 0 && c0 <= xmax - 1) {
    const long g = c0;
    r += ov3[((((piece_d(c0, k0, g) * 2 + d0) * 5 + piece_d(c1, k1, g)) * 2 + d1) * 5 +
                piece_d(c2, k2, g)) * 2 + d2];
  }
  return r;
}

__device__ __forceinline__ double node_d(long x, long c, long k, int d) {
  return (k == d) ? (double)(x == c) : 0.0;
}

__device__ __forceinline__ double rt_inv(const RTParams &rt, double r) {
  switch (rt.kind) {
    case kRTChebyshev: return -(acos((r - rt.p0) / (r + rt.p0)) / rt.p1) + rt.npoint;
    case kRTPower: return pow(r / rt.p0, 1.0 / rt.p1) - 1;
    case kRTLinear: return (r - rt.p0) / rt.p1;
    case kRTExp: return log(r / rt.p0) / rt.p1;
    case kRTShiftedExp: return log((r + rt.p1) / rt.p0) / rt.p2;
    default: return r;
  }
}

// ------------------------------------------------------------------ project
// proj[s][lm] = sum_j g[s][j] Y[j][lm] / sigma[s] * sqrt(4 pi (2l + 1)) per atom,
// g[s][j] = rho wb w at the atom's point (shell s, direction j): a small GEMM
// (nrad x nang) x (nang x lsize) on the FP64 tensor pipe (DMMA m16n8k8).
// g is first formed once per point into the plan's scratch P.pg (project_g_kernel),
// so that both operands stream straight from memory: CTA = (64 lm, 64 shells,
// atom x solve), 4 warps of 32 shells x 32 lm; the directions run in chunks of
// 16 through a kProjStages-deep cp.async ring in shared memory (g as
// [shell][j], Y as [j][lm], row strides = 4 mod 16 doubles so that each
// half-warp's fragment loads hit 16 distinct banks), each chunk's loads issued
// kProjStages - 1 chunks ahead of its products.
constexpr int kProjTile = 64, kProjK = 16, kProjThreads = 128, kProjStages = 3;
constexpr int kProjLda = kProjK + 4, kProjLdb = kProjTile + 4;
constexpr int kProjPer = kProjTile * kProjK / kProjThreads;  // copies per thread per chunk
constexpr size_t kProjStageDoubles = kProjTile * kProjLda + kProjK * kProjLdb;

// pg[solve][p] = rho wb w at every point of every atom (the same product, in
// the same order, the projection used to form per element).
__global__ void project_g_kernel(PoissonDev P, const double *__restrict__ rho,
                                 const double *__restrict__ wb,
                                 const double *__restrict__ w) {
  const int bat = blockIdx.y / P.natom;
  const PoissonAtom &at = P.atoms[blockIdx.y - bat * P.natom];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= at.nrad * at.nang) return;
  const long p = at.point_off + i;
  P.pg[bat * P.pg_stride + p] = rho[bat * P.batch_ld + p] * wb[p] * w[p];
}

__device__ __forceinline__ void proj_copy8(double *dst, const double *src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(valid ? 8 : 0)
               : "memory");
}

__global__ void __launch_bounds__(kProjThreads, 3) project_kernel(PoissonDev P) {
  extern __shared__ __align__(16) double psm[];
  const int bat = blockIdx.z / P.natom;  // solve of a batch
  const PoissonAtom at = P.atoms[blockIdx.z - bat * P.natom];
  const double *g = P.pg + bat * P.pg_stride;
  double *proj = P.proj + bat * P.proj_stride;
  const int lsize = (at.lmax + 1) * (at.lmax + 1);
  const int lm0 = blockIdx.x * kProjTile, s0 = blockIdx.y * kProjTile;
  if (lm0 >= lsize || s0 >= at.nrad) return;
  const int nang = at.nang, nrad = at.nrad;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int gq = lane >> 2, q = lane & 3;
  const int wr = (wid >> 1) * 32, wc = (wid & 1) * 32;  // warp tile origin
  const double *Y = P.ytab + at.ytab_off;
  const int nchunk = (nang + kProjK - 1) / kProjK;
  // chunk c into ring stage c % kProjStages (zero outside the atom's table)
  auto issue = [&](int c) {
    double *as = psm + (c % kProjStages) * kProjStageDoubles;
    double *bs = as + kProjTile * kProjLda;
    const int j0 = c * kProjK;
#pragma unroll
    for (int r = 0; r < kProjPer; ++r) {
      const int e = t + r * kProjThreads;
      {
        const int sl = e / kProjK, jj = e % kProjK;
        const int sh = s0 + sl, j = j0 + jj;
        const bool ok = sh < nrad && j < nang;
        proj_copy8(as + sl * kProjLda + jj, ok ? g + at.point_off + (long)sh * nang + j : g, ok);
      }
      {
        const int jj = e / kProjTile, ll = e % kProjTile;
        const int j = j0 + jj, lm = lm0 + ll;
        const bool ok = j < nang && lm < lsize;
        proj_copy8(bs + jj * kProjLdb + ll, ok ? Y + (long)j * lsize + lm : Y, ok);
      }
    }
  };
  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][k][c] = 0.0;
#pragma unroll
  for (int c = 0; c < kProjStages - 1; ++c) {
    if (c < nchunk) issue(c);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int c = 0; c < nchunk; ++c) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kProjStages - 2) : "memory");
    __syncthreads();  // chunk c is in for every thread; stage (c - 1) is free
    if (c + kProjStages - 1 < nchunk) issue(c + kProjStages - 1);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    const double *as = psm + (c % kProjStages) * kProjStageDoubles;
    const double *bs = as + kProjTile * kProjLda;
#pragma unroll
    for (int kk = 0; kk < kProjK; kk += 8) {
      double a[2][4], b[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const double *ar = as + (wr + mt * 16 + gq) * kProjLda + kk + q;
        a[mt][0] = ar[0];
        a[mt][1] = ar[8 * kProjLda];
        a[mt][2] = ar[4];
        a[mt][3] = ar[8 * kProjLda + 4];
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const double *br = bs + (kk + q) * kProjLdb + wc + nt * 8 + gq;
        b[nt][0] = br[0];
        b[nt][1] = br[4 * kProjLdb];
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], a[mt], b[nt]);
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  const double *sigma = P.rad + at.rad_off + kRadSigma * nrad;
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int lm = lm0 + wc + nt * 8 + 2 * q + c;
      if (lm >= lsize) continue;
      const int l = (int)sqrt((double)lm + 0.5);
      const double fac = sqrt(4.0 * M_PI * (2.0 * l + 1));
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int sh = s0 + wr + mt * 16 + gq + 8 * h;
          if (sh < nrad)
            proj[at.proj_off + (long)sh * lsize + lm] = acc[mt][nt][2 * h + c] / sigma[sh] * fac;
        }
      }
    }
  }
}

// ------------------------------------------------------------------- radial
// Band storage of the 2n x 2n FEM matrix (kKL, kKU, kW in poisson.cuh):
// AB(i, j) = band[j*kW + 6+i-j].

__device__ __forceinline__ double &AB(double *band, int i, int j) {
  return band[j * kW + (kKL + kKU) + i - j];
}

// The FEM band matrix of a system depends on the atom's radial grid and l
// only: it is assembled and LU-factored (partial pivoting, kl = ku = 3) once
// per grid.  Outputs per system: the band with U (rows i, columns i..i+6), the
// multipliers of step k in mult[k * kKL + i], the pivot row of step k.
// Thomas sweep of the (2 1 / 1 4 1 / ... / 1 2) cubic-spline system with the
// atom's precomputed denominators: t-derivatives dt of the spline through y
// (strides ys, ds), the same operations as the Poisson radial kernel's.
__device__ void spline_dt_col(const double *y, int ys, double *dt, int ds,
                              const double *den, const double *upm, int n) {
  double prev = (3.0 * (y[ys] - y[0])) / den[0];
  dt[0] = prev;
  for (int i = 1; i < n; ++i) {
    const double rhs = (i < n - 1) ? 3.0 * (y[(i + 1) * ys] - y[(i - 1) * ys])
                                   : 3.0 * (y[(n - 1) * ys] - y[(n - 2) * ys]);
    prev = (rhs - prev * 1.0) / den[i];
    dt[i * ds] = prev;
  }
  for (int i = n - 2; i >= 0; --i) dt[i * ds] = dt[i * ds] - upm[i] * dt[(i + 1) * ds];
}

// CTA = one radial system (atom, l): assembles the Hermite FEM band matrix of
// u'' + b u' + a u and factors it.  Poisson: a = -l(l+1)/r^2 (analytic
// derivative); Becke-Dickson (op.vsph set): a tabulated on the radial points
// with its spline derivative (ndpsi.py:58-69).
__global__ void radial_factor_kernel(PoissonDev P, RadialOp op) {
  extern __shared__ double sm[];
  const int sys = blockIdx.x;
  const PoissonAtom at = P.atoms[P.sys_atom[sys]];
  const int l = P.sys_l[sys];
  const int n = at.nrad, n2 = 2 * n;
  const int tid = threadIdx.x, nt = blockDim.x;
  double *band = sm;          // n2 * kW
  double *ay = band + n2 * kW;  // Becke-Dickson a(r_i) and its spline t-derivative
  double *adt = ay + n;
  __shared__ double s_mult[kKL];
  __shared__ double s_ov2[5 * 2 * 5 * 2], s_ov3[5 * 2 * 5 * 2 * 5 * 2];
  for (int e = threadIdx.x; e < 100; e += blockDim.x) s_ov2[e] = c_ov2[e];
  for (int e = threadIdx.x; e < 1000; e += blockDim.x) s_ov3[e] = c_ov3[e];
  const double *rad = P.rad + at.rad_off;
  const double *r = rad + kRadR * n, *j1 = rad + kRadJ1 * n, *j2 = rad + kRadJ2 * n,
               *j3 = rad + kRadJ3 * n;
  const long xmax = n - 1;
  double *lu = P.lu + (long)sys * P.lu_stride * kW;
  double *mult = P.lmul + (long)sys * P.lu_stride * kKL;
  int *piv = P.lpiv + (long)sys * P.lu_stride;
  // -- 2. band matrix (depends on l only)
  for (int e = tid; e < n2 * kW; e += nt) band[e] = 0.0;
  const double l2l = (double)(l * (l + 1));
  const bool bd = op.vsph != nullptr;
  if (bd) {
    const double *vs = op.vsph + at.rad_off / kRadSlots;
    for (int i = tid; i < n; i += nt)
      ay[i] = op.ascale * (l2l * (1.0 / (r[i] * r[i])) + ((vs[i] - op.e) - op.de));
    __syncthreads();
    if (tid == 0) spline_dt_col(ay, 1, adt, 1, rad + kRadDen * n, rad + kRadUp * n, n);
  }
  __syncthreads();
  for (int row = tid; row < n2; row += nt) {
    if (row == 0 || row == n2 - 2) {
      AB(band, row, row) = 1.0;
      continue;
    }
    long lo = 2 * (row / 2 - 1), hi = 2 * (row / 2 + 2);
    if (lo < 0) lo = 0;
    if (hi > n2) hi = n2;
    // the coefficient functions b, a at the row's (at most 6) FEM functions
    // k, shared by all of its columns
    double bks[6], aks[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      const long k = lo + t;
      double bk = 0.0, ak = 0.0;
      if (k < hi) {
        const int i = (int)(k / 2);
        const double ri = r[i], r2 = ri * ri;
        const double jsq = j1[i] * j1[i];
        if (bd) {
          // b = (2 r^-1, -2 r^-2) as ndpsi.py:55 forms it
          const double rinv = 1.0 / ri, r2inv = 1.0 / r2;
          if ((k & 1) == 0) {
            bk = j1[i] * (2.0 * rinv) - j2[i] / j1[i];
            ak = ay[i] * jsq;
          } else {
            bk = j2[i] * (2.0 * rinv) + jsq * (-2.0 * r2inv) +
                 (j2[i] * j2[i] - j1[i] * j3[i]) / jsq;
            const double adx = adt[i] / j1[i];
            ak = (adx * jsq + 2 * ay[i] * j2[i]) * j1[i];
          }
        } else if ((k & 1) == 0) {
          bk = j1[i] * (2 / ri) - j2[i] / j1[i];
          ak = (-l2l / r2) * jsq;
        } else {
          bk = j2[i] * (2 / ri) + jsq * (-2 / r2) + (j2[i] * j2[i] - j1[i] * j3[i]) / jsq;
          const double ay = -l2l / r2, adx = 2 * l2l / (r2 * ri);
          ak = (adx * jsq + 2 * ay * j2[i]) * j1[i];
        }
      }
      bks[t] = bk;
      aks[t] = ak;
    }
    for (long col = lo; col < hi; ++col) {
      double cf = 0.0;
      cf -= ov2_d(xmax, row, 1, col, 1, s_ov2);
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const long k = lo + t;
        if (k >= hi) break;
        const double bk = bks[t], ak = aks[t];
        if (bk != 0) cf += bk * ov3_d(xmax, row, 0, col, 1, k, 0, s_ov3);
        if (ak != 0) cf += ak * ov3_d(xmax, row, 0, col, 0, k, 0, s_ov3);
      }
      cf += node_d(xmax, row / 2, row % 2, 0) * node_d(xmax, col / 2, col % 2, 1);
      cf -= node_d(0, row / 2, row % 2, 0) * node_d(0, col / 2, col % 2, 1);
      AB(band, row, (int)col) = cf;
    }
  }
  __syncthreads();
  // -- 3. banded LU with partial pivoting.  A step updates at most 3 x 9
  // entries, so warp 0 runs the elimination with warp-level synchronisation
  // (a block barrier per step, 2 n times, cost more than the step itself).
  if (tid < 32) {
    const unsigned full = 0xffffffffu;
    for (int k = 0; k < n2; ++k) {
      const int im = min(k + kKL, n2 - 1);
      const int ju = min(k + kKL + kKU, n2 - 1);
      int p = k;
      if (tid == 0) {
        double best = fabs(AB(band, k, k));
        for (int i = k + 1; i <= im; ++i) {
          const double v = fabs(AB(band, i, k));
          if (v > best) {
            best = v;
            p = i;
          }
        }
      }
      p = __shfl_sync(full, p, 0);
      if (p != k) {
        for (int j = k + tid; j <= ju; j += 32) {
          const double t = AB(band, k, j);
          AB(band, k, j) = AB(band, p, j);
          AB(band, p, j) = t;
        }
        __syncwarp();
      }
      if (tid < im - k) s_mult[tid] = AB(band, k + 1 + tid, k) / AB(band, k, k);
      __syncwarp();
      const int nrow = im - k, ncolu = ju - k;
      for (int e = tid; e < nrow * ncolu; e += 32) {
        const int i = k + 1 + e / ncolu, j = k + 1 + e % ncolu;
        AB(band, i, j) -= s_mult[i - k - 1] * AB(band, k, j);
      }
      if (tid == 0) {
        piv[k] = p;
        for (int i = 0; i < kKL; ++i) mult[k * kKL + i] = i < nrow ? s_mult[i] : 0.0;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int e = tid; e < n2 * kW; e += nt) lu[e] = band[e];
}

// Radial solve.  CTA = (system (atom, l), group of solves of the batch);
// thread = one column (solve, m), lm = l^2 + m.  A column is a chain of
// dependent steps: the Thomas sweep of the spline through f_lm (with the
// boundary moments), the forward elimination of the FEM right-hand side with
// the system's LU factors, and the back substitution, whose values leave as
// spline tables.  Each step of a chain is one FMA on the chained value
// (divisions become products with reciprocals tabulated when the CTA stages
// its tables; the back substitution uses U's rows scaled by 1/U_ii).  Each
// sweep keeps its live rows in registers (a window of 4 rows forward, 6 back)
// and hands its results to the next through the column's scratch in global
// memory, laid out [slot][lm] per (solve, atom) so that a warp's accesses are
// contiguous (slots [0, n): t-derivatives, [n, 3n): eliminated rows).  A sweep
// reads its global inputs through a per-thread ring in shared memory filled by
// cp.async kRing - 2 steps ahead (L2 latency would otherwise stall each step,
// and a register ring needs unrolled code); a slot is refilled two steps after
// it was read.  The right-hand side of a row is
// assembled as the forward sweep reaches it, from the three nodes around it.
// Shared memory also holds the system's factors, the atom's radial tables and
// the Hermite overlaps of every row with the 6 functions of its nodes q - 1 ..
// q + 1 (q = row / 2; 0 where a node does not exist).  The arithmetic is that
// of poisson_solver.py:42-118 and ode2.py (spline, FEM assembly, banded LU
// solve with partial pivoting), up to rounding.
constexpr int kRadialThreads = 128;
constexpr int kRing = 32;  // doubles per thread: one ring of 32 or two of 16

__host__ __device__ __forceinline__ size_t radial_smem_bytes(int n, int threads) {
  const size_t n2 = 2 * (size_t)n;
  return (n2 * (6 + kKL + 6 + 1) + 7 * (size_t)n + (size_t)kRing * threads) * sizeof(double) +
         n2 * sizeof(int);
}

// solves per CTA of `threads` threads for a system with 2l + 1 columns
__host__ __device__ __forceinline__ int radial_solves_per_cta(int l, int threads) {
  const int s = threads / (2 * l + 1);
  return s > 0 ? s : 1;
}

__device__ __forceinline__ void ring_copy(double *dst, const double *src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void ring_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void ring_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(kRadialThreads) radial_kernel(PoissonDev P, RadialOp op) {
  extern __shared__ double sm[];
  const int sys = blockIdx.x;
  const PoissonAtom at = P.atoms[P.sys_atom[sys]];
  const int l = P.sys_l[sys];
  const int ncol = 2 * l + 1, spc = radial_solves_per_cta(l, blockDim.x);
  const int bat0 = blockIdx.y * spc;
  if (bat0 >= P.nbatch) return;  // the whole CTA
  const int n = at.nrad, n2 = 2 * n;
  const int lsize = (at.lmax + 1) * (at.lmax + 1);
  const long xmax = n - 1;
  const int tid = threadIdx.x, nt = blockDim.x;
  double *ub = sm;                // [n2][6]: U_i,i+1..i+6 / U_ii
  double *rU = ub + 6 * n2;       // [n2]: 1 / U_ii
  double *mult = rU + n2;         // [n2][kKL]
  double *ovr = mult + n2 * kKL;  // [n2][6]
  double *j1 = ovr + 6 * n2, *j2 = j1 + n, *rj1 = j2 + n, *rden = rj1 + n, *upm = rden + n,
         *rlw = upm + n, *rmw = rlw + n;
  double *ring = rmw + n;  // [kRing][nt]
  int *piv = reinterpret_cast<int *>(ring + kRing * nt);
  {
    const double *gb = P.lu + (long)sys * P.lu_stride * kW;
    const double *gm = P.lmul + (long)sys * P.lu_stride * kKL;
    const int *gp = P.lpiv + (long)sys * P.lu_stride;
    // band storage: AB(i, j) = gb[j kW + kKL + kKU + i - j]
    for (int i = tid; i < n2; i += nt) {
      const double d = 1.0 / gb[i * kW + kKL + kKU];
      rU[i] = d;
      for (int t = 1; t <= kKL + kKU; ++t)
        ub[6 * i + t - 1] = i + t < n2 ? gb[(i + t) * kW + kKL + kKU - t] * d : 0.0;
      piv[i] = gp[i];
    }
    for (int e = tid; e < n2 * kKL; e += nt) mult[e] = gm[e];
    const double *rad = P.rad + at.rad_off;
    for (int i = tid; i < n; i += nt) {
      const double r = rad[kRadR * n + i], w = rad[kRadW * n + i];
      j1[i] = rad[kRadJ1 * n + i];
      j2[i] = rad[kRadJ2 * n + i];
      rj1[i] = 1.0 / j1[i];
      rden[i] = 1.0 / rad[kRadDen * n + i];
      upm[i] = rad[kRadUp * n + i];
      rlw[i] = pow(r, (double)l) * w;
      rmw[i] = pow(r, (double)(-l - 1)) * w;
    }
    for (int e = tid; e < 6 * n2; e += nt) {
      const int row = e / 6, t = e - 6 * row;
      const long k = 2 * (long)(row / 2 - 1) + t;
      long lo = 2 * (row / 2 - 1), hi = 2 * (row / 2 + 2);
      if (lo < 0) lo = 0;
      if (hi > n2) hi = n2;
      ovr[e] = (k >= lo && k < hi) ? ov2_d(xmax, row, 0, k, 0) : 0.0;
    }
  }
  __syncthreads();
  const int sidx = tid / ncol, m = tid - sidx * ncol;
  const long bat = bat0 + sidx;
  if (sidx >= spc || bat >= P.nbatch) return;  // no barrier below
  const int lm = l * l + m;
  const int ls = lsize;
  const double *Y = P.proj + bat * P.proj_stride + at.proj_off + lm;  // f_lm(r_i) at Y[i ls]
  double *S = P.rscr + bat * P.rscr_stride + at.scr_off + lm;        // slot s at S[s ls]
  double *E = S + n * ls;                                             // eliminated rows
  double *q = ring + tid;  // this thread's ring: slot s at q[s nt]
  constexpr int R1 = kRing, R2 = kRing / 2;  // ring lengths; lookahead R - 2
  auto back2 = [](int slot, int R) { return slot >= 2 ? slot - 2 : slot + R - 2; };
  double *qa = q, *qb = q + R2 * nt;  // two rings of R2 for the forward elimination

  // -- 1. spline t-derivatives of f_lm (Thomas elimination of 2/1, 1/4/1,
  // ..., 1/2 with rhs 3 (y_{i+1} - y_{i-1})) and the radial moments of the
  // Dirichlet values.  Step i (1 <= i < n) reads y_{i+1} from ring slot i % R1.
  const bool moments = !op.zero_bc;
  double smax = 0.0, smin = 0.0, prev;
  {
    for (int s = 1; s < R1 - 1; ++s) {
      ring_copy(q + s * nt, Y + (s + 1 < n ? s + 1 : 0) * ls, s + 1 < n);
      ring_commit();
    }
    double ym = Y[0], yc = Y[ls];
    prev = (3.0 * (yc - ym)) * rden[0];
    S[0] = prev;
    if (moments) {
      smax = ym * rlw[0];
      smin = ym * rmw[0];
    }
    int slot = 1;
    for (int i = 1; i < n; ++i) {
      const int j = i + R1 - 1;  // y index the refill brings, for step i + R1 - 2
      ring_copy(q + back2(slot, R1) * nt, Y + (j < n ? j : 0) * ls, j < n);
      ring_commit();
      ring_wait<R1 - 2>();
      const double yn = q[slot * nt];
      slot = slot + 1 == R1 ? 0 : slot + 1;
      const double rhs = (i < n - 1) ? 3.0 * (yn - ym) : 3.0 * (yc - ym);
      prev = fma(-prev, rden[i], rhs * rden[i]);
      S[i * ls] = prev;
      if (moments) {
        smax = fma(yc, rlw[i], smax);
        smin = fma(yc, rmw[i], smin);
      }
      ym = yc;
      yc = yn;
    }
    ring_wait<0>();
  }
  __threadfence_block();  // the stores above before the ring's reads below
  {
    // step t reads prev_i, i = n - 2 - t, from slot t % R1
    for (int t = 0; t < R1 - 2; ++t) {
      const int i = n - 2 - t;
      ring_copy(q + t * nt, S + (i >= 0 ? i : 0) * ls, i >= 0);
      ring_commit();
    }
    double dn = prev;  // dt[n - 1]
    int slot = 0;
    for (int t = 0; t < n - 1; ++t) {
      const int i = n - 2 - t, j = i - (R1 - 2);  // the refill is for step t + R1 - 2
      ring_copy(q + back2(slot, R1) * nt, S + (j >= 0 ? j : 0) * ls, j >= 0);
      ring_commit();
      ring_wait<R1 - 2>();
      const double pn = q[slot * nt];
      slot = slot + 1 == R1 ? 0 : slot + 1;
      dn = fma(-upm[i], dn, pn);
      S[i * ls] = dn;
    }
    ring_wait<0>();
  }
  double bcmin = 0.0, bcmax = 0.0;
  if (moments) {
    const double *rad = P.rad + at.rad_off;
    bcmax = smax / (pow(rad[kRadR * n + n - 1], (double)(l + 1)) * (2 * l + 1));
    bcmin = smin * (pow(rad[kRadR * n], (double)l) / (2 * l + 1));
  }
  __threadfence_block();

  // -- 2. FEM right-hand side (source f = fscale f_lm) row by row, eliminated
  // with the factors as it is assembled.  Node i contributes fe = fy j1^2 to
  // the sums of even rows and fo = (fdx j1^2 + 2 fy j2) j1 to odd ones
  // (fy = fscale f_lm(r_i), fdx = fscale dt_i / j1_i).
  const double fs = op.fscale;
  auto node_f = [&](int i, double y, double dt, double &fe, double &fo) {
    if (i >= n) {
      fe = fo = 0.0;
      return;
    }
    const double fy = fs * y;
    const double jsq = j1[i] * j1[i];
    fe = fy * jsq;
    fo = fma(fs * (dt * rj1[i]), jsq, 2 * fy * j2[i]) * j1[i];
  };
  // nodes q - 1, q, q + 1 of the rows 2q, 2q + 1 being assembled
  double ae = 0.0, ao = 0.0, be, bo, ce, co;
  auto rhs_row = [&](int row) -> double {
    if (row == 0) return bcmin;
    if (row == n2 - 2) return bcmax;
    if (row >= n2) return 0.0;
    const double *o = ovr + 6 * row;
    double acc = ae * o[0];
    acc = fma(ao, o[1], acc);
    acc = fma(be, o[2], acc);
    acc = fma(bo, o[3], acc);
    acc = fma(ce, o[4], acc);
    return fma(co, o[5], acc);
  };
  node_f(0, Y[0], S[0], be, bo);
  node_f(1, Y[ls], S[ls], ce, co);
  double w0 = rhs_row(0), w1 = rhs_row(1), w2, w3;  // rows k .. k + 3
  ae = be;
  ao = bo;
  be = ce;
  bo = co;
  node_f(2, n > 2 ? Y[2 * ls] : 0.0, n > 2 ? S[2 * ls] : 0.0, ce, co);
  w2 = rhs_row(2);
  w3 = rhs_row(3);
  auto step = [&](int k) {
    const int d = piv[k] - k;
    const double m0 = mult[k * kKL], m1 = mult[k * kKL + 1], m2 = mult[k * kKL + 2];
    const double t0 = w0;
    w0 = d == 1 ? w1 : (d == 2 ? w2 : (d == 3 ? w3 : w0));
    w1 = d == 1 ? t0 : w1;
    w2 = d == 2 ? t0 : w2;
    w3 = d == 3 ? t0 : w3;
    const double rk = w0;
    w1 = fma(-m0, rk, w1);
    w2 = fma(-m1, rk, w2);
    w3 = fma(-m2, rk, w3);
    E[k * ls] = rk;
    w0 = w1;
    w1 = w2;
    w2 = w3;
  };
  {
    // iteration it brings in node it + 3: (f_lm, dt) from slot it % R2 of
    // the two rings
    for (int s = 0; s < R2 - 2; ++s) {
      const int i = s + 3;
      ring_copy(qa + s * nt, Y + (i < n ? i : 0) * ls, i < n);
      ring_copy(qb + s * nt, S + (i < n ? i : 0) * ls, i < n);
      ring_commit();
    }
    int slot = 0;
    for (int it = 0; it < n; ++it) {
      const int k = 2 * it, i = it + 3 + (R2 - 2);  // node of the refill
      const int rs = back2(slot, R2);
      ring_copy(qa + rs * nt, Y + (i < n ? i : 0) * ls, i < n);
      ring_copy(qb + rs * nt, S + (i < n ? i : 0) * ls, i < n);
      ring_commit();
      step(k);
      ring_wait<R2 - 2>();
      const double yv = qa[slot * nt], dv = qb[slot * nt];
      slot = slot + 1 == R2 ? 0 : slot + 1;
      ae = be;
      ao = bo;
      be = ce;
      bo = co;
      node_f(it + 3, yv, dv, ce, co);
      w3 = rhs_row(k + 4);
      step(k + 1);
      w3 = rhs_row(k + 5);
    }
    ring_wait<0>();
  }
  __threadfence_block();

  // -- 3. back substitution, x_i = E_i / U_ii - sum_j (U_ij / U_ii) x_j;
  // node j's values (rows 2j, 2j + 1) leave as the cubic of interval j (scaled
  // by sqrt(2l+1)/sqrt(4 pi)), raw (y, dy/dt) and the extrapolation amplitudes.
  // Step t handles row i = n2 - 1 - t, E_i from slot t % R1.
  const double fl = sqrt((double)(2 * l + 1)) * kInvSqrt4Pi;
  double *spl = P.spl + bat * P.spl_stride + at.spl_off + (long)lm * 4;
  double *amp = P.amp + bat * P.amp_stride + at.amp_off + lm * 2;
  double x1 = 0.0, x2 = 0.0, x3 = 0.0, x4 = 0.0, x5 = 0.0, x6 = 0.0;  // rows i + 1 .. i + 6
  double dnext = 0.0;  // dy/dt of node j + 1
  for (int t = 0; t < R1 - 2; ++t) {
    const int i = n2 - 1 - t;
    ring_copy(q + t * nt, E + (i >= 0 ? i : 0) * ls, i >= 0);
    ring_commit();
  }
  int slot = 0;
  for (int i = n2 - 1; i >= 0; --i) {
    const int j = i - (R1 - 2);
    ring_copy(q + back2(slot, R1) * nt, E + (j >= 0 ? j : 0) * ls, j >= 0);
    ring_commit();
    ring_wait<R1 - 2>();
    const double ei = q[slot * nt];
    slot = slot + 1 == R1 ? 0 : slot + 1;
    const double *ui = ub + 6 * i;  // zero beyond the last row
    double x = ei * rU[i];
    x = fma(-ui[5], x6, x);
    x = fma(-ui[4], x5, x);
    x = fma(-ui[3], x4, x);
    x = fma(-ui[2], x3, x);
    x = fma(-ui[1], x2, x);
    x = fma(-ui[0], x1, x);
    if ((i & 1) == 0) {
      const int jn = i / 2;
      const double d0 = (x1 * rj1[jn]) * j1[jn];
      if (P.raw_y) {
        const long o = at.raw_off + (long)lm * n + jn;
        P.raw_y[o] = x;
        P.raw_dt[o] = d0;
      }
      if (jn < n - 1) {
        const double z = x2 - x;
        double *cf = spl + (long)jn * lsize * 4;
        cf[0] = x * fl;
        cf[1] = d0 * fl;
        cf[2] = (3 * z - 2 * d0 - dnext) * fl;
        cf[3] = (-2 * z + d0 + dnext) * fl;
      } else {
        amp[1] = x * pow(at.last_x, (double)(l + 1)) * fl;
      }
      if (i == 0) amp[0] = x / pow(at.first_x, (double)l) * fl;
      dnext = d0;
    }
    x6 = x5;
    x5 = x4;
    x4 = x3;
    x3 = x2;
    x2 = x1;
    x1 = x;
  }
  ring_wait<0>();
}

// ------------------------------------------------------------------ kinetic
// CTA = (system (atom, l), chunk of ncol columns m).  Per column: the radial
// operator (1/r d2/dr2 r - l(l+1)/r^2) f_lm by finite differences in the
// Chebyshev angle w (r = radii (1 + cos w)/(1 - cos w), w_i = (i + 1) pi /
// (n + 1) belongs to radial point n - 1 - i), then the cubic spline of the
// result with the potential extrapolation (nkinetic.py:48-61,
// src/grid/radial.cpp:51-192), scaled by `scale` into the evaluation tables.
__global__ void kinetic_radial_kernel(PoissonDev P, int ncol, double scale) {
  extern __shared__ double sm[];
  const int sys = blockIdx.x;
  const PoissonAtom at = P.atoms[P.sys_atom[sys]];
  const int l = P.sys_l[sys];
  const int n = at.nrad;
  const int lsize = (at.lmax + 1) * (at.lmax + 1);
  const int c0 = blockIdx.y * ncol;
  if (c0 >= 2 * l + 1) return;
  const int nm = min(ncol, 2 * l + 1 - c0);
  const int tid = threadIdx.x, nt = blockDim.x;
  double *Y = sm;            // n * ncol: projected function, then spline t-derivatives
  double *V = Y + n * ncol;  // n * ncol: operator values
  double *r = V + n * ncol, *den = r + n, *upm = den + n;
  {
    const double *rad = P.rad + at.rad_off;
    for (int i = tid; i < n; i += nt) {
      r[i] = rad[kRadR * n + i];
      den[i] = rad[kRadDen * n + i];
      upm[i] = rad[kRadUp * n + i];
    }
    const double *proj = P.proj + at.proj_off + l * l + c0;
    for (int e = tid; e < n * nm; e += nt) {
      const int i = e / nm, c = e - i * nm;
      Y[i * ncol + c] = proj[(long)i * lsize + c];
    }
  }
  __syncthreads();
  const double radii = at.rt.p0, H = M_PI / (n + 1.0), l2l = (double)(l * (l + 1));
  for (int e = tid; e < n * nm; e += nt) {
    const int idx = e / nm, c = e - idx * nm;
    const int i = n - 1 - idx;
    const double *g = Y + c;  // g(k) = f(w_k) = g[(n - 1 - k) * ncol]
    double d1 = 0.0, d2 = 0.0;
    if (i < 4) {
      for (int k = 0; k < 7; ++k) {
        const double gk = g[(n - 1 - k) * ncol];
        d1 += c_fd[i * 7 + k] * gk;
        d2 += c_fd[28 + i * 7 + k] * gk;
      }
      d1 /= c_fd[74] * H;
      d2 /= c_fd[75] * H * H;
    } else if (i >= n - 4) {
      const int j = n - 1 - i;  // mirror of edge node j: first-derivative weights change sign
      for (int k = 6; k >= 0; --k) {
        const double gk = g[k * ncol];  // f(w_(n-1-k))
        d1 -= c_fd[j * 7 + k] * gk;
        d2 += c_fd[28 + j * 7 + k] * gk;
      }
      d1 /= c_fd[74] * H;
      d2 /= c_fd[75] * H * H;
    } else {
      for (int k = 0; k < 9; ++k) {
        const double gk = g[(n - 1 - (i - 4 + k)) * ncol];
        d1 += c_fd[56 + k] * gk;
        d2 += c_fd[65 + k] * gk;
      }
      d1 /= c_fd[76] * H;
      d2 /= c_fd[77] * H * H;
    }
    // dw/dr and d2w/dr2 of the Chebyshev map
    const double w = (i + 1) * H, X = cos(w), Yw = sin(w), q = 1.0 - X;
    const double wr = -q * q / (2.0 * radii * Yw);
    const double wrr = q * q * q * (2.0 * Yw * Yw - q * X) / (4.0 * radii * radii * Yw * Yw * Yw);
    const double ri = r[idx];
    const double lap = wr * wr * d2 + (wrr + 2.0 * wr / ri) * d1;
    V[idx * ncol + c] = lap - l2l * (1.0 / (ri * ri)) * Y[idx * ncol + c];
  }
  __syncthreads();
  for (int c = tid; c < nm; c += nt) spline_dt_col(V + c, ncol, Y + c, ncol, den, upm, n);
  __syncthreads();
  const double fl = sqrt((double)(2 * l + 1)) * kInvSqrt4Pi * scale;
  for (int e = tid; e < (n - 1) * nm; e += nt) {
    const int j = e / nm, c = e - j * nm;
    const double y0 = V[j * ncol + c], y1 = V[(j + 1) * ncol + c];
    const double d0 = Y[j * ncol + c], d1 = Y[(j + 1) * ncol + c];
    const double z = y1 - y0;
    double *cf = P.spl + at.spl_off + ((long)j * lsize + l * l + c0 + c) * 4;
    cf[0] = y0 * fl;
    cf[1] = d0 * fl;
    cf[2] = (3 * z - 2 * d0 - d1) * fl;
    cf[3] = (-2 * z + d0 + d1) * fl;
  }
  for (int c = tid; c < nm; c += nt) {
    const int lm = l * l + c0 + c;
    P.amp[at.amp_off + lm * 2 + 0] = V[c] / pow(at.first_x, (double)l) * fl;
    P.amp[at.amp_off + lm * 2 + 1] = V[(n - 1) * ncol + c] * pow(at.last_x, (double)(l + 1)) * fl;
  }
}

// One warp per (radial shell, atom): sum_j f wb w / sum_j w over the shell.
__global__ void __launch_bounds__(32)
shell_average_kernel(PoissonDev P, const double *__restrict__ f, const double *__restrict__ wb,
                     const double *__restrict__ w, double *__restrict__ out) {
  const PoissonAtom at = P.atoms[blockIdx.y];
  const int sh = blockIdx.x;
  if (sh >= at.nrad) return;
  const long base = at.point_off + (long)sh * at.nang;
  double acc = 0.0;
  for (int j = threadIdx.x; j < at.nang; j += 32) acc += f[base + j] * wb[base + j] * w[base + j];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (threadIdx.x == 0)
    out[at.rad_off / kRadSlots + sh] = acc / P.rad[at.rad_off + kRadSigma * at.nrad + sh];
}

// ----------------------------------------------------------------- evaluate
template <int LMAX>
__global__ void __launch_bounds__(128)
evaluate_kernel(PoissonDev P, int npoint, const double *__restrict__ gx,
                const double *__restrict__ gy, const double *__restrict__ gz,
                double *__restrict__ out, int accumulate) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  int mol = 0;
  if (P.nmol > 1) {
    int lo = 0, hi = P.nmol - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.mol_point_off[mid] <= p) lo = mid; else hi = mid - 1;
    }
    mol = lo;
  }
  const double px = gx[p], py = gy[p], pz = gz[p];
  double v = accumulate ? out[p] : 0.0;
  const int a1 = P.mol_atom_off[mol + 1];
  for (int A = P.mol_atom_off[mol]; A < a1; ++A) {
    const PoissonAtom &at = P.atoms[A];
    const double dx = px - at.cx, dy = py - at.cy, dz = pz - at.cz;
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    const int lmaxA = at.lmax;
    const int lsize = (lmaxA + 1) * (lmaxA + 1);
    int region;  // 0 spline, 1 left tail, 2 right tail
    const double *cf = nullptr;
    const double *amp = P.amp + at.amp_off;
    double u = 0.0;
    if (d < at.first_x) {
      region = 1;
    } else if (d <= at.last_x) {
      region = 0;
      const double t = rt_inv(at.rt, d);
      int j = (int)floor(t);
      if (j == at.nrad - 1) j = at.nrad - 2;
      if (j < 0) j = 0;
      u = t - j;
      cf = P.spl + at.spl_off + (long)j * lsize * 4;
    } else {
      region = 2;
    }
    double dl = 1.0;  // d^l for the tails
    auto sval = [&](int lm) -> double {
      if (region == 0) {
        const double2 c01 = __ldg(reinterpret_cast<const double2 *>(cf + lm * 4));
        const double2 c23 = __ldg(reinterpret_cast<const double2 *>(cf + lm * 4 + 2));
        return c01.x + u * (c01.y + u * (c23.x + u * c23.y));
      }
      if (region == 1) return amp[lm * 2] * dl;
      return amp[lm * 2 + 1] / (dl * d);
    };
    v += sval(0);
    if (LMAX >= 1 && lmaxA >= 1) {
      const double dinv = 1.0 / d;
      double dpowl = dinv;
      dl = d;
      v += sval(1) * dpowl * dz;
      v += sval(2) * dpowl * dx;
      v += sval(3) * dpowl * dy;
      if (LMAX >= 2 && lmaxA >= 2) {
        const double r2 = dx * dx + dy * dy + dz * dz;
        double pold[LMAX + 1], pnew[LMAX + 1], cs[LMAX + 1], sn[LMAX + 1];
        pold[0] = 1.0;
        pnew[0] = dz;
        pnew[1] = 1.0;
        cs[1] = dx;
        sn[1] = dy;
        int lm = 4;
#pragma unroll
        for (int l = 2; l <= LMAX; ++l) {
          if (l > lmaxA) break;
          dpowl *= dinv;
          dl *= d;
          const double fac = 2 * l - 1;
#pragma unroll
          for (int m = 0; m <= l - 2; ++m) {
            const double keep = pold[m];
            pold[m] = pnew[m];
            pnew[m] = (dz * fac * pold[m] - r2 * (l + m - 1) * keep) * (1.0 / (l - m));
          }
          pold[l - 1] = pnew[l - 1];
          pnew[l] = fac * pold[l - 1];
          pnew[l - 1] = dz * pnew[l];
          cs[l] = dx * cs[l - 1] - dy * sn[l - 1];
          sn[l] = dx * sn[l - 1] + dy * cs[l - 1];
          v += sval(lm) * dpowl * pnew[0];
          ++lm;
#pragma unroll
          for (int m = 1; m <= l; ++m) {
            const double nrm = c_shnorm[l * (kMaxLmax + 1) + m];
            v += sval(lm) * dpowl * (nrm * cs[m] * pnew[m]);
            v += sval(lm + 1) * dpowl * (nrm * sn[m] * pnew[m]);
            lm += 2;
          }
        }
      }
    }
  }
  out[p] = v;
}

// --------------------------------------------------- bucketed evaluation
// Bucket of the pair (atom A, point p): 0 below the first radial point, 1 + j
// inside spline interval j, nrad above the last point -- the same region and
// interval test as the spline evaluation of the reference
// (src/horton/cubic_spline.cpp:147-181).
__device__ __forceinline__ int pair_bucket(const PoissonAtom &at, double px, double py,
                                           double pz) {
  const double dx = px - at.cx, dy = py - at.cy, dz = pz - at.cz;
  const double d = sqrt(dx * dx + dy * dy + dz * dz);
  if (d < at.first_x) return 0;
  if (d > at.last_x) return at.nrad;
  int j = (int)floor(rt_inv(at.rt, d));
  if (j == at.nrad - 1) j = at.nrad - 2;
  if (j < 0) j = 0;
  return 1 + j;
}

// Neighbouring points mostly fall in the same bucket of an atom, so the
// counters are bumped once per group of lanes with equal buckets (the lowest
// lane adds the group's size): one atomic per group instead of per pair.
__device__ __forceinline__ int lanes_below(unsigned m) {
  return __popc(m & ((1u << (threadIdx.x & 31)) - 1u));
}

__global__ void pair_bucket_kernel(PoissonDev P, const double *__restrict__ gx,
                                   const double *__restrict__ gy,
                                   const double *__restrict__ gz, const int *__restrict__ keep,
                                   int *__restrict__ bucket_of, int *__restrict__ count) {
  const PoissonAtom &at = P.atoms[blockIdx.y];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = q < at.mol_npoint;
  int b = -1;
  if (in) {
    const int p = at.mol_point_start + q;
    if (!keep || keep[p]) b = pair_bucket(at, gx[p], gy[p], gz[p]);  // -1: screened out
    bucket_of[at.pair_off + q] = b;
  }
  const unsigned group = __match_any_sync(0xffffffffu, b);
  if (b >= 0 && lanes_below(group) == 0) atomicAdd(&count[at.bucket_off + b], __popc(group));
}

// Distance of point p from the atom, as the evaluation computes it.
__device__ __forceinline__ double pair_distance(const PoissonAtom &at, const double *gx,
                                                const double *gy, const double *gz, int p) {
  const double dx = gx[p] - at.cx, dy = gy[p] - at.cy, dz = gz[p] - at.cz;
  return sqrt(dx * dx + dy * dy + dz * dz);
}

__global__ void pair_scatter_kernel(PoissonDev P, const double *__restrict__ gx,
                                    const double *__restrict__ gy,
                                    const double *__restrict__ gz,
                                    const int *__restrict__ bucket_of,
                                    int *__restrict__ cursor) {
  const PoissonAtom &at = P.atoms[blockIdx.y];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = q < at.mol_npoint ? bucket_of[at.pair_off + q] : -1;
  const unsigned group = __match_any_sync(0xffffffffu, b);
  const int leader = __ffs(group) - 1;
  int base = 0;
  if (b >= 0 && (int)(threadIdx.x & 31) == leader)
    base = atomicAdd(&cursor[at.bucket_off + b], __popc(group));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (b >= 0) {
    const long slot = at.pair_off + base + lanes_below(group);
    const int p = at.mol_point_start + q;
    P.pairs[slot] = p;
    if (b > 0 && b < at.nrad) {  // interior: the evaluation's u and 1/d
      const double d = pair_distance(at, gx, gy, gz, p);
      P.pair_u[slot] = make_double2(rt_inv(at.rt, d) - (b - 1), 1.0 / d);
    }
  }
}

// One CTA per EvalItem: the coefficient block of the item's spline interval
// (or the tail amplitudes) is staged in shared memory once and every thread
// evaluates one pair:
//   v_pair = sum_k u^k sum_lm S_lm(r_hat) c_k,lm        (interval)
//   v_pair = sum_l g_l(d) sum_m S_lm(r_hat) a_lm         (tails, g = d^l or
//                                                         d^-(l+1))
// with S_lm(r_hat) = S_lm(p - A) / d^l, so the 1/d^l of the reference is folded
// into the unit vector.  The result goes to the pair's own slot of pair_v.
// Potentials of NP (atom, point) pairs of one bucket from the shared
// coefficients cf (each coefficient load serves all NP pairs): REGION 0
// inside the atom's radial grid (cubic spline in the interval coordinate u),
// 1 below its first point (amplitudes x d^l), 2 beyond its last (amplitudes
// x d^-(l+1)).
template <int LMAX, int REGION, int NP>
__device__ __forceinline__ void pair_values(const double *cf, int lmaxA, const double *x,
                                            const double *y, const double *z, const double *d,
                                            const double *inv, const double *u, double *v) {
  double a0[NP], a1[NP], a2[NP], a3[NP], gstep[NP], cm[NP], sm[NP], gm[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    a0[j] = a1[j] = a2[j] = a3[j] = 0.0;
    // tail factor of the current l: 1 inside the grid, d^l below its first
    // point, d^-(l+1) beyond its last
    gstep[j] = REGION == 1 ? d[j] : (REGION == 2 ? inv[j] : 1.0);
    gm[j] = REGION == 2 ? inv[j] : 1.0;
    cm[j] = 1.0;
    sm[j] = 0.0;
  }
  // accumulate the (lm, S) term of every pair
  auto term = [&](int lm, const double *S, const double *gl) {
    if (REGION == 0) {
      const double2 c01 = *reinterpret_cast<const double2 *>(cf + 4 * lm);
      const double2 c23 = *reinterpret_cast<const double2 *>(cf + 4 * lm + 2);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        a0[j] = fma(c01.x, S[j], a0[j]);
        a1[j] = fma(c01.y, S[j], a1[j]);
        a2[j] = fma(c23.x, S[j], a2[j]);
        a3[j] = fma(c23.y, S[j], a3[j]);
      }
    } else {
      const double c = cf[lm];
#pragma unroll
      for (int j = 0; j < NP; ++j) a0[j] = fma(c * gl[j], S[j], a0[j]);
    }
  };
  // Normalised solid harmonics of the unit vector, m outer and l inner:
  // q_l^m = nrm_lm Pi_l^m with Pi_m^m = (2m-1)!!, Pi_(m+1)^m = (2m+1) z Pi_m^m,
  // Pi_l^m = ((2l-1) z Pi_(l-1)^m - (l+m-1) Pi_(l-2)^m) / (l-m) (|u| = 1);
  // the normalisation is folded into the recursion constants (c_rec_a,
  // c_rec_start) and the recursion runs on q~ = q / gamma (c_rec_gamma), whose
  // scale the staged coefficients carry.  S_l0 = q_l^0; S_lm (cos, sin) =
  // q_l^m Re/Im (x + iy)^m at lm = l^2 + 2m - 1, l^2 + 2m: the values and lm
  // order of solid_harmonics.h, evaluated column by column so that only a few
  // are live.
#pragma unroll
  for (int m = 0; m <= LMAX; ++m) {
    if (m > lmaxA) break;
    double q[NP], qprev[NP], gl[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      if (m > 0) {
        const double c = cm[j] * x[j] - sm[j] * y[j];
        sm[j] = cm[j] * y[j] + sm[j] * x[j];
        cm[j] = c;
        gm[j] *= gstep[j];
      }
      q[j] = c_rec_start[m];
      qprev[j] = 0.0;
      gl[j] = gm[j];
    }
#pragma unroll
    for (int l = m; l <= LMAX; ++l) {
      if (l > lmaxA) break;
      if (l > m) {
        const int k = l * (kMaxLmax + 1) + m;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          const double qn = fma(c_rec_a[k], z[j] * q[j], -qprev[j]);
          qprev[j] = q[j];
          q[j] = qn;
          gl[j] *= gstep[j];
        }
      }
      if (m == 0) {
        term(l * l, q, gl);
      } else {
        double sc[NP], ss[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          sc[j] = q[j] * cm[j];
          ss[j] = q[j] * sm[j];
        }
        term(l * l + 2 * m - 1, sc, gl);
        term(l * l + 2 * m, ss, gl);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NP; ++j)
    v[j] = REGION == 0 ? a0[j] + u[j] * (a1[j] + u[j] * (a2[j] + u[j] * a3[j])) : a0[j];
}


// max over 0 <= u <= 1 of |c0 + c1 u + c2 u^2 + c3 u^3|: the ends and the
// interior zeros of the derivative (stable quadratic roots), plus 1e-12 of
// sum_k |c_k| for the rounding of the evaluation and of the roots.
__device__ double cubic_max_abs(const double *c) {
  auto val = [&](double u) { return c[0] + u * (c[1] + u * (c[2] + u * c[3])); };
  double m = fmax(fabs(c[0]), fabs(val(1.0)));
  const double a = 3.0 * c[3], b = 2.0 * c[2], cc = c[1];
  if (a != 0.0) {
    const double disc = b * b - 4.0 * a * cc;
    if (disc >= 0.0) {
      const double h = -0.5 * (b + copysign(sqrt(disc), b));
      const double r1 = h / a, r2 = h != 0.0 ? cc / h : r1;
      if (r1 > 0.0 && r1 < 1.0) m = fmax(m, fabs(val(r1)));
      if (r2 > 0.0 && r2 < 1.0) m = fmax(m, fabs(val(r2)));
    }
  } else if (b != 0.0) {
    const double r = -cc / b;
    if (r > 0.0 && r < 1.0) m = fmax(m, fabs(val(r)));
  }
  return m + 1e-12 * (fabs(c[0]) + fabs(c[1]) + fabs(c[2]) + fabs(c[3]));
}

// Truncation of the expansion per (atom, bucket) when P.eval_tol > 0.  With
// Racah-normalised harmonics sum_m S_lm(r_hat)^2 = 1, so by Cauchy-Schwarz the
// l-block adds at most bound_l = sqrt(sum_m c_lm^2) to the potential of any
// pair of the bucket, with c_lm = max |U_lm(u)| over the interval's cubic
// (0 <= u <= 1) inside the grid, |a_lm| first_x^l below the first radial point
// (d^l <= first_x^l) and |a_lm| last_x^-(l+1) beyond the last.  The bucket
// keeps l <= L, the smallest L whose dropped blocks sum to at most eval_tol.
// Grid (max nrad + 1, natom), one warp: the lanes bound the (l, m) terms
// lane, lane + 32, ... (every lane busy, whatever l), then lane l sums block l
// in m order.
__global__ void __launch_bounds__(32) bucket_lcut_kernel(PoissonDev P) {
  __shared__ double bound[32];
  extern __shared__ double cterm[];  // (max_lmax + 1)^2
  const int bat = blockIdx.y / P.natom;  // solve of a batch
  const PoissonAtom &at = P.atoms[blockIdx.y - bat * P.natom];
  const double *const spl = P.spl + bat * P.spl_stride;
  const double *const amp = P.amp + bat * P.amp_stride;
  const int b = blockIdx.x, l = threadIdx.x;
  if (b > at.nrad) return;
  const int lmaxA = at.lmax;
  const int lsize = (lmaxA + 1) * (lmaxA + 1);
  const int region = (b == 0) ? 1 : (b == at.nrad ? 2 : 0);
  for (int lm = l; lm < lsize; lm += 32)
    cterm[lm] = region == 0 ? cubic_max_abs(spl + at.spl_off + ((long)(b - 1) * lsize + lm) * 4)
                            : fabs(amp[at.amp_off + lm * 2 + (region == 1 ? 0 : 1)]);
  __syncwarp();
  if (l <= lmaxA) {
    double s2 = 0.0;
    for (int lm = l * l; lm < (l + 1) * (l + 1); ++lm) s2 = fma(cterm[lm], cterm[lm], s2);
    const double g = region == 0 ? 1.0
                                 : (region == 1 ? pow(at.first_x, (double)l)
                                                : pow(at.last_x, -(double)(l + 1)));
    bound[l] = sqrt(s2) * g;
  }
  __syncwarp();
  if (l == 0) {
    double dropped = 0.0;
    int L = lmaxA;
    while (L > 0 && dropped + bound[L] <= P.eval_tol) dropped += bound[L--];
    P.lcut[bat * P.lcut_stride + at.bucket_off + b] = L;
  }
}

// TAILS = false: the interior items [0, nitems_inner) (region 0 only, so the
// kernel carries that region's code alone); true: the others.
// BATCH: the launch evaluates several solves (blockIdx.y); the single-solve
// instance carries no batch offsets (its registers, and occupancy, stay those
// the recursion was tuned at)
template <int LMAX, bool TAILS, bool BATCH>
// Four 256-thread CTAs per SM (64 registers, 20 bytes spilled): 32 resident
// warps instead of 24 at the compiler's 76 registers; the FP64 pipe, busy 77 %
// at 24 warps, throttles less often (C20H42 evaluation 3 % faster).
__global__ void __launch_bounds__(kEvalChunkMax / kEvalPerThread, 4)
eval_pairs_kernel(PoissonDev P, const double *__restrict__ gx,
                  const double *__restrict__ gy, const double *__restrict__ gz) {
  extern __shared__ double cf[];
  const EvalItem it = P.items[blockIdx.x + (TAILS ? P.nitems_inner : 0)];
  const PoissonAtom &at = P.atoms[it.atom];
  const int lmaxA = at.lmax;
  const int lsize = (lmaxA + 1) * (lmaxA + 1);
  const int region = TAILS ? (it.bucket == 0 ? 1 : 2) : 0;
  const long bat = BATCH ? (long)blockIdx.y : 0;  // solve of a batch
  // l-blocks kept for this bucket (all unless a truncation tolerance is set)
  const int lcut = P.lcut ? P.lcut[bat * P.lcut_stride + at.bucket_off + it.bucket] : lmaxA;
  const int lkeep = (lcut + 1) * (lcut + 1);
  // staged with the recursion's scale gamma_lm (see c_rec_gamma)
  if (region == 0) {
    const double *src =
        P.spl + bat * P.spl_stride + at.spl_off + (long)(it.bucket - 1) * lsize * 4;
    for (int e = threadIdx.x; e < lkeep * 4; e += blockDim.x) cf[e] = src[e] * g_rec_gamma[e >> 2];
  } else {
    const double *src = P.amp + bat * P.amp_stride + at.amp_off;
    for (int e = threadIdx.x; e < lkeep; e += blockDim.x)
      cf[e] = src[2 * e + (region == 1 ? 0 : 1)] * g_rec_gamma[e];
  }
  __syncthreads();
  // thread t evaluates the pairs t and t + blockDim.x of the item (the
  // second may be absent: it then repeats the first and is not stored)
  const int t = threadIdx.x;
  if (t >= it.count) return;
  int pidx[kEvalPerThread];
  double x[kEvalPerThread], y[kEvalPerThread], z[kEvalPerThread], d[kEvalPerThread],
      inv[kEvalPerThread], u[kEvalPerThread], v[kEvalPerThread];
#pragma unroll
  for (int j = 0; j < kEvalPerThread; ++j) {
    const int e = t + j * (int)blockDim.x;
    const long slot = at.pair_off + it.start + (e < it.count ? e : t);
    pidx[j] = P.pairs[slot];
    const int p = pidx[j];
    const double dx = gx[p] - at.cx, dy = gy[p] - at.cy, dz = gz[p] - at.cz;
    if (region == 0) {  // u and 1/d stored with the pair lists
      const double2 ui = P.pair_u[slot];
      u[j] = ui.x;
      inv[j] = ui.y;
      d[j] = 0.0;  // unused inside the grid
    } else {
      d[j] = pair_distance(at, gx, gy, gz, p);
      inv[j] = 1.0 / d[j];
      u[j] = 0.0;
    }
    x[j] = dx * inv[j];
    y[j] = dy * inv[j];
    z[j] = dz * inv[j];
  }
  if (!TAILS)
    pair_values<LMAX, 0, kEvalPerThread>(cf, lcut, x, y, z, d, inv, u, v);
  else if (region == 1)
    pair_values<LMAX, 1, kEvalPerThread>(cf, lcut, x, y, z, d, inv, u, v);
  else
    pair_values<LMAX, 2, kEvalPerThread>(cf, lcut, x, y, z, d, inv, u, v);
#pragma unroll
  for (int j = 0; j < kEvalPerThread; ++j) {
    const int e = t + j * (int)blockDim.x;
    if (e < it.count)
      P.pair_v[bat * P.pairv_stride + at.pair_off + (pidx[j] - at.mol_point_start)] = v[j];
  }
}

// v[p] (+)= sum over the atoms of p's molecule of pair_v, in atom order.
__global__ void pairs_reduce_kernel(PoissonDev P, int npoint, double *__restrict__ out,
                                    int accumulate) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  const int bat = blockIdx.y;  // solve of a batch
  out += bat * P.batch_ld;
  const double *pair_v = P.pair_v + bat * P.pairv_stride;
  if (P.keep && !P.keep[p]) {  // screened-out point: no potential evaluated
    if (!accumulate) out[p] = 0.0;
    return;
  }
  int mol = 0;
  if (P.nmol > 1) {
    int lo = 0, hi = P.nmol - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.mol_point_off[mid] <= p) lo = mid; else hi = mid - 1;
    }
    mol = lo;
  }
  double v = accumulate ? out[p] : 0.0;
  const int a1 = P.mol_atom_off[mol + 1];
  for (int A = P.mol_atom_off[mol]; A < a1; ++A) {
    const PoissonAtom &at = P.atoms[A];
    v += pair_v[at.pair_off + (p - at.mol_point_start)];
  }
  out[p] = v;
}

template <int L>
cudaError_t launch_eval_l(const PoissonDev &P, int npoint, const double *x,
                          const double *y, const double *z, double *out, int acc,
                          cudaStream_t s) {
  if (P.items && P.nitems > 0) {
    if (P.lcut) {
      bucket_lcut_kernel<<<dim3(P.max_nrad + 1, P.natom * P.nbatch), 32,
                           (size_t)(P.max_lmax + 1) * (P.max_lmax + 1) * sizeof(double), s>>>(P);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
    const size_t smem = (size_t)(L + 1) * (L + 1) * 4 * sizeof(double);
    const dim3 gin(P.nitems_inner, P.nbatch), gtail(P.nitems - P.nitems_inner, P.nbatch);
    const int kT = P.eval_chunk / kEvalPerThread;
    if (P.nitems_inner > 0) {
      if (P.nbatch > 1)
        eval_pairs_kernel<L, false, true><<<gin, kT, smem, s>>>(P, x, y, z);
      else
        eval_pairs_kernel<L, false, false><<<gin, kT, smem, s>>>(P, x, y, z);
    }
    if (P.nitems > P.nitems_inner) {
      if (P.nbatch > 1)
        eval_pairs_kernel<L, true, true><<<gtail, kT, smem, s>>>(P, x, y, z);
      else
        eval_pairs_kernel<L, true, false><<<gtail, kT, smem, s>>>(P, x, y, z);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pairs_reduce_kernel<<<dim3((npoint + 255) / 256, P.nbatch), 256, 0, s>>>(P, npoint, out,
                                                                             acc);
    return cudaGetLastError();
  }
  if (P.nbatch != 1) return cudaErrorInvalidValue;  // batches need the pair lists
  evaluate_kernel<L><<<(npoint + 127) / 128, 128, 0, s>>>(P, npoint, x, y, z, out, acc);
  return cudaGetLastError();
}

}  // namespace

// Uploads the constant tables to the current device.  Called by every Poisson
// plan construction (which allocates and copies far more): uploading per plan
// rather than once per device keeps the tables in place under any context and
// after a device reset.  The bytes are the same every time, so an upload while
// kernels of another plan read the tables changes nothing they see.
cudaError_t poisson_init_constants() {
  cudaError_t e = cudaSuccess;
  std::vector<double> ov2(100), ov3(1000);
  hermite_tables_export(ov2.data(), ov3.data());
  std::vector<double> nrm((kMaxLmax + 1) * (kMaxLmax + 1), 0.0);
  for (int l = 1; l <= kMaxLmax; ++l) {
    double f = M_SQRT2;
    for (int m = 1; m <= l; ++m) {
      f /= sqrt((double)((l + m) * (l - m + 1)));
      nrm[l * (kMaxLmax + 1) + m] = f;
    }
  }
  if ((e = cudaMemcpyToSymbol(c_ov2, ov2.data(), ov2.size() * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_ov3, ov3.data(), ov3.size() * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_shnorm, nrm.data(), nrm.size() * sizeof(double))) != cudaSuccess) return e;
  {
    const int K = kMaxLmax + 1;
    auto nr = [&](int l, int m) { return m == 0 ? 1.0 : nrm[l * K + m]; };
    std::vector<double> ra(K * K, 0.0), rb(K * K, 0.0), st(K, 0.0);
    double dfact = 1.0;  // (2m-1)!!
    for (int m = 0; m <= kMaxLmax; ++m) {
      if (m > 0) dfact *= (double)(2 * m - 1);
      st[m] = nr(m, m) * dfact;
      for (int l = m + 1; l <= kMaxLmax; ++l) {
        if (l == m + 1) {
          ra[l * K + m] = (double)(2 * m + 1) * nr(l, m) / nr(m, m);
        } else {
          ra[l * K + m] = (double)(2 * l - 1) / (double)(l - m) * nr(l, m) / nr(l - 1, m);
          rb[l * K + m] = (double)(l + m - 1) / (double)(l - m) * nr(l, m) / nr(l - 2, m);
        }
      }
    }
    // rescaled recursion: gamma per (l, m), A = a gamma_(l-1) / gamma_l, and
    // gamma laid out per lm (cos and sin columns share it)
    std::vector<double> gam(K * K, 1.0), A(K * K, 0.0), gam_lm(K * K, 1.0);
    for (int m = 0; m <= kMaxLmax; ++m)
      for (int l = m; l <= kMaxLmax; ++l) {
        if (l >= m + 2) gam[l * K + m] = rb[l * K + m] * gam[(l - 2) * K + m];
        if (l > m) A[l * K + m] = ra[l * K + m] * gam[(l - 1) * K + m] / gam[l * K + m];
        if (m == 0) {
          gam_lm[l * l] = gam[l * K];
        } else {
          gam_lm[l * l + 2 * m - 1] = gam[l * K + m];
          gam_lm[l * l + 2 * m] = gam[l * K + m];
        }
      }
    if ((e = cudaMemcpyToSymbol(c_rec_a, A.data(), A.size() * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_rec_gamma, gam_lm.data(), gam_lm.size() * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_rec_start, st.data(), st.size() * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_rec_gamma, gam_lm.data(), gam_lm.size() * sizeof(double))) !=
        cudaSuccess)
      return e;
  }
  {
    const Deriv2Stencils &st = deriv2_stencils();
    double fd[78];
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 7; ++k) {
        fd[j * 7 + k] = st.edge1[j][k];
        fd[28 + j * 7 + k] = st.edge2[j][k];
      }
    for (int k = 0; k < 9; ++k) {
      fd[56 + k] = st.mid1[k];
      fd[65 + k] = st.mid2[k];
    }
    fd[74] = st.den_edge1;
    fd[75] = st.den_edge2;
    fd[76] = st.den_mid1;
    fd[77] = st.den_mid2;
    if ((e = cudaMemcpyToSymbol(c_fd, fd, sizeof(fd))) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_poisson_project(const PoissonDev &P, const double *rho,
                                   const double *wb, const double *w,
                                   cudaStream_t s) {
  if (P.natom == 0) return cudaSuccess;
  if (!P.pg) return cudaErrorInvalidValue;
  const int maxpts = P.max_nrad * P.max_nang;
  project_g_kernel<<<dim3((maxpts + 255) / 256, P.natom * P.nbatch), 256, 0, s>>>(P, rho, wb,
                                                                                 w);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int lsize = (P.max_lmax + 1) * (P.max_lmax + 1);
  dim3 grid((lsize + kProjTile - 1) / kProjTile, (P.max_nrad + kProjTile - 1) / kProjTile,
            P.natom * P.nbatch);
  constexpr size_t smem = kProjStages * kProjStageDoubles * sizeof(double);
  e = cudaFuncSetAttribute(project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) return e;
  project_kernel<<<grid, kProjThreads, smem, s>>>(P);
  return cudaGetLastError();
}

constexpr size_t kMaxSmem = 227 * 1024;

size_t poisson_factor_doubles(int nsys, int max_nrad) {
  return (size_t)nsys * 2 * max_nrad * (kW + kKL);
}

cudaError_t launch_radial_factor(const PoissonDev &P, const RadialOp &op, cudaStream_t s) {
  if (P.nsys == 0) return cudaSuccess;
  const size_t smem =
      ((size_t)2 * P.max_nrad * kW + (op.vsph ? 2 * (size_t)P.max_nrad : 0)) * sizeof(double);
  // static part: the Hermite tables and the multipliers
  constexpr size_t kStatic = (100 + 1000 + kKL) * sizeof(double);
  if (smem + kStatic > kMaxSmem) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(radial_factor_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // 4 warps: rows of the assembly in parallel; the elimination is one chain
  radial_factor_kernel<<<P.nsys, 128, smem, s>>>(P, op);
  return cudaGetLastError();
}

cudaError_t launch_poisson_factor(const PoissonDev &P, cudaStream_t s) {
  return launch_radial_factor(P, RadialOp(), s);
}

cudaError_t launch_radial_solve(const PoissonDev &P, const RadialOp &op, cudaStream_t s) {
  if (P.nsys == 0) return cudaSuccess;
  // one warp per CTA for single solves (idle lanes' shared memory would limit
  // the CTAs per SM), up to kRadialThreads for batches; the CTAs of a system
  // take radial_solves_per_cta(l, threads) solves each, and the grid's y
  // covers the batch for the largest l (CTAs past it return)
  const long cols = (long)(2 * P.max_lmax + 1) * P.nbatch;
  const int threads = (int)std::min<long>(kRadialThreads, (cols + 31) / 32 * 32);
  const size_t smem = radial_smem_bytes(P.max_nrad, threads);
  if (smem > kMaxSmem || 2 * P.max_lmax + 1 > kRadialThreads || !P.rscr)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(radial_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int spc = radial_solves_per_cta(P.max_lmax, threads);
  const int groups = (P.nbatch + spc - 1) / spc;
  radial_kernel<<<dim3(P.nsys, groups), threads, smem, s>>>(P, op);
  return cudaGetLastError();
}

cudaError_t launch_poisson_radial(const PoissonDev &P, cudaStream_t s) {
  return launch_radial_solve(P, RadialOp(), s);
}

cudaError_t launch_kinetic_radial(const PoissonDev &P, double scale, cudaStream_t s) {
  if (P.nsys == 0) return cudaSuccess;
  const size_t n = (size_t)P.max_nrad;
  int ncol = 32;
  while (ncol > 1 && (2 * n * ncol + 3 * n) * sizeof(double) > kMaxSmem) ncol /= 2;
  const size_t smem = (2 * n * ncol + 3 * n) * sizeof(double);
  if (smem > kMaxSmem) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(kinetic_radial_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int nchunk = (2 * P.max_lmax + 1 + ncol - 1) / ncol;
  kinetic_radial_kernel<<<dim3(P.nsys, nchunk), 128, smem, s>>>(P, ncol, scale);
  return cudaGetLastError();
}

cudaError_t launch_shell_average(const PoissonDev &P, const double *f, const double *wb,
                                 const double *w, double *out, cudaStream_t s) {
  if (P.natom == 0) return cudaSuccess;
  shell_average_kernel<<<dim3(P.max_nrad, P.natom), 32, 0, s>>>(P, f, wb, w, out);
  return cudaGetLastError();
}

cudaError_t launch_pair_buckets(const PoissonDev &P, int max_mol_npoint, const double *x,
                                const double *y, const double *z, const int *keep,
                                int *bucket_of, int *count, cudaStream_t s) {
  dim3 grid((max_mol_npoint + 255) / 256, P.natom);
  pair_bucket_kernel<<<grid, 256, 0, s>>>(P, x, y, z, keep, bucket_of, count);
  return cudaGetLastError();
}

cudaError_t launch_pair_scatter(const PoissonDev &P, int max_mol_npoint, const double *x,
                                const double *y, const double *z, const int *bucket_of,
                                int *cursor, cudaStream_t s) {
  dim3 grid((max_mol_npoint + 255) / 256, P.natom);
  pair_scatter_kernel<<<grid, 256, 0, s>>>(P, x, y, z, bucket_of, cursor);
  return cudaGetLastError();
}

cudaError_t launch_poisson_evaluate(const PoissonDev &P, int npoint,
                                    const double *x, const double *y,
                                    const double *z, double *out, bool accumulate,
                                    cudaStream_t s) {
  if (npoint <= 0) return cudaSuccess;
  const int a = accumulate ? 1 : 0;
  switch (P.max_lmax) {
#define NAPMO_EVAL_CASE(L) \
  case L: return launch_eval_l<L>(P, npoint, x, y, z, out, a, s);
    NAPMO_EVAL_CASE(0) NAPMO_EVAL_CASE(1) NAPMO_EVAL_CASE(2) NAPMO_EVAL_CASE(3)
    NAPMO_EVAL_CASE(4) NAPMO_EVAL_CASE(5) NAPMO_EVAL_CASE(6) NAPMO_EVAL_CASE(7)
    NAPMO_EVAL_CASE(8) NAPMO_EVAL_CASE(9) NAPMO_EVAL_CASE(10) NAPMO_EVAL_CASE(11)
    NAPMO_EVAL_CASE(12) NAPMO_EVAL_CASE(13) NAPMO_EVAL_CASE(14) NAPMO_EVAL_CASE(15)
    NAPMO_EVAL_CASE(16) NAPMO_EVAL_CASE(17) NAPMO_EVAL_CASE(18) NAPMO_EVAL_CASE(19)
    NAPMO_EVAL_CASE(20)
#undef NAPMO_EVAL_CASE
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace napmo
