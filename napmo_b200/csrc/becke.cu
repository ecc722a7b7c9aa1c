// Becke multicentre partition weights (A. D. Becke, J. Chem. Phys. 88, 2547
// (1988), eqs. 11, 19-22 and appendix A), bit-identical to nAPMO's OpenMP
// host loop (src/grid/becke.cpp:79-176).
//
// This translation unit is compiled with --fmad=false: every product and sum
// is rounded separately in the same order as the reference, and CUDA's double
// division and square root are IEEE round-to-nearest, so each weight matches
// the reference bit for bit.
//
// Layout: one thread per grid point.  The atom origins, the packed R_ij /
// a_ij triangles and the per-atom point offsets live in shared memory (in
// global memory, read as warp-wide broadcasts, above ~130 centres); each
// thread's distances r_A to all atoms are cached in a shared column
// [atom][thread] (bank-conflict free), computed once instead of once per
// pair.  The owner atom of a point is found from the per-atom offsets, so
// atomic grids of different sizes are handled (the reference assumes equal
// sizes and indexes atom * (size / ncenter) + point, which agrees whenever
// the sizes are equal).
#include "common.h"
#include "kernels.cuh"

namespace napmo {

namespace {

constexpr int kBeckeThreads = 128;

__device__ __forceinline__ double distance3(double px, double py, double pz,
                                            const double *o) {
  double acc = 0.0;
  double d = px - o[0];
  acc += d * d;
  d = py - o[1];
  acc += d * d;
  d = pz - o[2];
  acc += d * d;
  return sqrt(acc);
}

__device__ __forceinline__ int owner_of(int p, const int *off, int nc) {
  int lo = 0, hi = nc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= p) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Cell-function product p_i = prod_{j != i} s(nu_ij) and the final ratio.
// kSmem: the centre tables (origins, R_ij, a_ij, offsets) are staged in
// shared memory; without it (more centres than fit, about 130) they are read
// from global memory, where every lane of a warp reads the same address in
// the same order (one broadcast per load, L1-resident).  kCacheR: each
// thread's distances to all centres are cached in shared memory.  The
// arithmetic is the same in every variant.
template <bool kCacheR, bool kSmem>
__global__ void __launch_bounds__(kBeckeThreads)
becke_kernel(int npoint, int nc, const double *__restrict__ gx,
             const double *__restrict__ gy, const double *__restrict__ gz,
             const double *__restrict__ g_origin, const double *__restrict__ g_R,
             const double *__restrict__ g_a, const int *__restrict__ g_off,
             double *__restrict__ out) {
  extern __shared__ double smem[];
  const int tri = nc * (nc + 1) / 2;
  const double *s_origin = g_origin, *s_R = g_R, *s_a = g_a;
  const int *s_off = g_off;
  double *s_r = smem;                      // nc * blockDim (kCacheR)
  if (kSmem) {
    double *o = smem;                      // 3 * nc
    double *R = o + 3 * nc;                // tri
    double *a = R + tri;                   // tri
    s_r = a + tri;
    int *off = reinterpret_cast<int *>(s_r + (kCacheR ? nc * kBeckeThreads : 0));
    for (int i = threadIdx.x; i < 3 * nc; i += blockDim.x) o[i] = g_origin[i];
    for (int i = threadIdx.x; i < tri; i += blockDim.x) {
      R[i] = g_R[i];
      a[i] = g_a[i];
    }
    for (int i = threadIdx.x; i <= nc; i += blockDim.x) off[i] = g_off[i];
    __syncthreads();
    s_origin = o;
    s_R = R;
    s_a = a;
    s_off = off;
  }

  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  const double px = gx[p], py = gy[p], pz = gz[p];
  const int owner = owner_of(p, s_off, nc);

  if (kCacheR) {
    for (int i = 0; i < nc; ++i)
      s_r[i * kBeckeThreads + threadIdx.x] = distance3(px, py, pz, s_origin + 3 * i);
  }

  double sum = 0.0;
  double mine = 0.0;
  for (int i = 0; i < nc; ++i) {
    double prod = 1.0;
    const double ri = kCacheR ? s_r[i * kBeckeThreads + threadIdx.x]
                              : distance3(px, py, pz, s_origin + 3 * i);
    for (int j = 0; j < nc; ++j) {
      if (i == j) continue;
      const int off = (i < j) ? (j * (j + 1)) / 2 + i : (i * (i + 1)) / 2 + j;
      const double rj = kCacheR ? s_r[j * kBeckeThreads + threadIdx.x]
                                : distance3(px, py, pz, s_origin + 3 * j);
      const double mu = (ri - rj) / s_R[off];
      const double sgn = (i < j) ? -1.0 : 1.0;
      double s = mu + s_a[off] * (sgn * (1.0 - mu * mu));
      s = 0.5 * s * (3.0 - s * s);
      s = 0.5 * s * (3.0 - s * s);
      s = 0.5 * s * (3.0 - s * s);
      s = 0.5 * (1.0 - s);
      prod *= s;
    }
    if (i == owner) mine = prod;
    sum += prod;
  }
  out[p] = mine / sum;
}

}  // namespace

cudaError_t launch_becke_weights(int npoint, int ncenter, const double *x,
                                 const double *y, const double *z,
                                 const double *origin, const double *Rij,
                                 const double *aij, const int *atom_offset,
                                 double *out, cudaStream_t s) {
  if (npoint <= 0) return cudaSuccess;
  const size_t tri = (size_t)ncenter * (ncenter + 1) / 2;
  const size_t base = (3 * (size_t)ncenter + 2 * tri) * sizeof(double) +
                      ((size_t)ncenter + 1) * sizeof(int);
  const size_t cached = base + (size_t)ncenter * kBeckeThreads * sizeof(double);
  const size_t rcache = (size_t)ncenter * kBeckeThreads * sizeof(double);
  const size_t limit = 200 * 1024;
  const int blocks = (npoint + kBeckeThreads - 1) / kBeckeThreads;
  cudaError_t e = cudaSuccess;
  if (cached <= limit) {
    e = cudaFuncSetAttribute(becke_kernel<true, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cached);
    if (e != cudaSuccess) return e;
    becke_kernel<true, true><<<blocks, kBeckeThreads, cached, s>>>(
        npoint, ncenter, x, y, z, origin, Rij, aij, atom_offset, out);
  } else if (base <= limit) {
    e = cudaFuncSetAttribute(becke_kernel<false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)base);
    if (e != cudaSuccess) return e;
    becke_kernel<false, true><<<blocks, kBeckeThreads, base, s>>>(
        npoint, ncenter, x, y, z, origin, Rij, aij, atom_offset, out);
  } else if (rcache <= limit) {
    // tables from global memory, distances cached in shared memory
    e = cudaFuncSetAttribute(becke_kernel<true, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rcache);
    if (e != cudaSuccess) return e;
    becke_kernel<true, false><<<blocks, kBeckeThreads, rcache, s>>>(
        npoint, ncenter, x, y, z, origin, Rij, aij, atom_offset, out);
  } else {
    // any number of centres: tables from global memory, distances recomputed
    becke_kernel<false, false><<<blocks, kBeckeThreads, 0, s>>>(
        npoint, ncenter, x, y, z, origin, Rij, aij, atom_offset, out);
  }
  return cudaGetLastError();
}

}  // namespace napmo
