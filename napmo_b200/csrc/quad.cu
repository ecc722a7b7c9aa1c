// FP64 grid quadratures on CUDA cores (the plain FP64 path):
//
//   density     rho[p]     = sum_{mu,nu} phi[mu][p] D[mu][nu] phi[nu][p]
//   quadrature  F[mu][nu]  = sum_p phi[mu][p] wv[p] phi[nu][p]
//               (or sum_p phi[mu][p] wv[p] psi[nu][p] for a second operand psi,
//               upper triangle mirrored as nAPMO does for exchange)
//
// nAPMO computes the density point by point in Python (psi_hybrid.py:144-150)
// and the quadrature by materialising every orbital product
// Psi[n(n+1)/2][N] (src/wavefunction/nwavefunction.cpp:77-107,161-197).  Here
// both are register-tiled DFMA GEMMs over phi stored basis-major
// [n][ld] (ld a multiple of 128, zero padded):
//
//   * density: a CTA owns 128 points, sweeps 128-row blocks of mu, forms
//     T = D phi for the block in registers and folds it into the per-point
//     sum with phi[mu][p] in the epilogue; deterministic, no atomics.
//   * quadrature: split-K over points.  CTA (tile, chunk) accumulates one
//     128x128 upper-triangle tile of F over one chunk of points into a
//     workspace slot; a second kernel adds the chunks in fixed order and
//     writes both triangles, so F is exactly symmetric and bit-reproducible.
//
// Tiles: 128x128 per CTA, 256 threads, 8x8 doubles per thread (two 4x4
// quadrants 64 apart), K step 8, register-staged double buffering.
#include <string>

#include "common.h"
#include "kernels.cuh"

namespace napmo {

namespace {

constexpr int BM = 128, BN = 128, BK = 8, NT = 256;

struct TileSmem {
  double a[2][BK][BM];
  double b[2][BK][BN];
};

// acc[i][j] += sum_k As[k][row(i)] * Bs[k][col(j)] for one BK slice.
__device__ __forceinline__ void mma_slice(const double (*As)[BM],
                                          const double (*Bs)[BN], int tx, int ty,
                                          double acc[8][8]) {
#pragma unroll
  for (int k = 0; k < BK; ++k) {
    double a[8], b[8];
    const double2 a0 = *reinterpret_cast<const double2 *>(&As[k][ty * 4]);
    const double2 a1 = *reinterpret_cast<const double2 *>(&As[k][ty * 4 + 2]);
    const double2 a2 = *reinterpret_cast<const double2 *>(&As[k][64 + ty * 4]);
    const double2 a3 = *reinterpret_cast<const double2 *>(&As[k][64 + ty * 4 + 2]);
    const double2 b0 = *reinterpret_cast<const double2 *>(&Bs[k][tx * 4]);
    const double2 b1 = *reinterpret_cast<const double2 *>(&Bs[k][tx * 4 + 2]);
    const double2 b2 = *reinterpret_cast<const double2 *>(&Bs[k][64 + tx * 4]);
    const double2 b3 = *reinterpret_cast<const double2 *>(&Bs[k][64 + tx * 4 + 2]);
    a[0] = a0.x; a[1] = a0.y; a[2] = a1.x; a[3] = a1.y;
    a[4] = a2.x; a[5] = a2.y; a[6] = a3.x; a[7] = a3.y;
    b[0] = b0.x; b[1] = b0.y; b[2] = b1.x; b[3] = b1.y;
    b[4] = b2.x; b[5] = b2.y; b[6] = b3.x; b[7] = b3.y;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
}

__device__ __forceinline__ int row_of(int ty, int i) {
  return (i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4);
}

// ------------------------------------------------------------------ density
// Loads of one K slice (rows nu0..nu0+7):
//   A: As[k][m] = D[nu0+k][mu0+m]  (D symmetric, so rows of D are columns)
//   B: Bs[k][c] = phi[nu0+k][p0+c]
__global__ void __launch_bounds__(NT)
density_kernel(int n, int npoint, const double *__restrict__ phi, long ld,
               const double *__restrict__ D, double *__restrict__ rho) {
  __shared__ __align__(16) TileSmem sm;
  __shared__ double red[16][BN];
  const int t = threadIdx.x, tx = t % 16, ty = t / 16;
  const int p0 = blockIdx.x * BN;
  // load mapping: each thread loads 4 consecutive elements of one K row
  const int lk = t / 32, lc = (t % 32) * 4;
  double part[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) part[j] = 0.0;

  const int nkb = (n + BK - 1) / BK;
  for (int mu0 = 0; mu0 < n; mu0 += BM) {
    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;

    double ra[4], rb[4];
    auto gload = [&](int kb) {
      const int nu = kb * BK + lk;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int mu = mu0 + lc + q;
        ra[q] = (nu < n && mu < n) ? __ldg(D + (long)nu * n + mu) : 0.0;
      }
      if (nu < n) {
        const double2 v0 = __ldg(reinterpret_cast<const double2 *>(phi + (long)nu * ld + p0 + lc));
        const double2 v1 = __ldg(reinterpret_cast<const double2 *>(phi + (long)nu * ld + p0 + lc + 2));
        rb[0] = v0.x; rb[1] = v0.y; rb[2] = v1.x; rb[3] = v1.y;
      } else {
        rb[0] = rb[1] = rb[2] = rb[3] = 0.0;
      }
    };
    auto sstore = [&](int buf) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        sm.a[buf][lk][lc + q] = ra[q];
        sm.b[buf][lk][lc + q] = rb[q];
      }
    };
    gload(0);
    sstore(0);
    __syncthreads();
    for (int kb = 0; kb < nkb; ++kb) {
      const int cur = kb & 1;
      if (kb + 1 < nkb) gload(kb + 1);
      mma_slice(sm.a[cur], sm.b[cur], tx, ty, acc);
      if (kb + 1 < nkb) sstore(cur ^ 1);
      __syncthreads();
    }
    // epilogue: part[c] += sum_i T[mu_i][c] phi[mu_i][c]
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int mu = mu0 + row_of(ty, i);
      if (mu < n) {
        const double *prow = phi + (long)mu * ld + p0;
#pragma unroll
        for (int j = 0; j < 8; ++j) part[j] = fma(acc[i][j], __ldg(prow + row_of(tx, j)), part[j]);
      }
    }
  }
  // reduce the 16 row-groups (ty) sharing each column
#pragma unroll
  for (int j = 0; j < 8; ++j) red[ty][row_of(tx, j)] = part[j];
  __syncthreads();
  if (t < BN) {
    double s = 0.0;
#pragma unroll
    for (int r = 0; r < 16; ++r) s += red[r][t];
    if (p0 + t < npoint) rho[p0 + t] = s;
  }
}

// --------------------------------------------------------------- quadrature
__global__ void __launch_bounds__(NT)
quadrature_kernel(int n, int npoint_pad, const double *__restrict__ phi,
                  const double *__restrict__ phib, long ld,
                  const double *__restrict__ wv, int nblk, int chunk,
                  double *__restrict__ work) {
  __shared__ __align__(16) TileSmem sm;
  const int t = threadIdx.x, tx = t % 16, ty = t / 16;
  // upper-triangle tile index -> (mb, nb)
  int tile = blockIdx.x, mb = 0;
  {
    int rem = tile;
    while (rem >= nblk - mb) {
      rem -= nblk - mb;
      ++mb;
    }
    tile = rem;  // offset within row mb
  }
  const int nb = mb + tile;
  const int mu0 = mb * BM, nu0 = nb * BN;
  const int k_begin = blockIdx.y * chunk;
  const int k_end = min(k_begin + chunk, npoint_pad);
  // load mapping: thread loads 4 consecutive k of one row (rows t/2, k (t%2)*4)
  const int lr = t / 2, lk = (t % 2) * 4;
  const int mu_l = mu0 + lr, nu_l = nu0 + lr;
  const double *arow = phi + (long)min(mu_l, n - 1) * ld;
  const double *brow = phib + (long)min(nu_l, n - 1) * ld;
  const bool aval = mu_l < n, bval = nu_l < n;

  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;

  double ra[4], rb[4];
  auto gload = [&](int k0) {
    const int k = k0 + lk;
    if (aval) {
      const double2 v0 = __ldg(reinterpret_cast<const double2 *>(arow + k));
      const double2 v1 = __ldg(reinterpret_cast<const double2 *>(arow + k + 2));
      ra[0] = v0.x; ra[1] = v0.y; ra[2] = v1.x; ra[3] = v1.y;
    } else {
      ra[0] = ra[1] = ra[2] = ra[3] = 0.0;
    }
    if (bval) {
      const double2 v0 = __ldg(reinterpret_cast<const double2 *>(brow + k));
      const double2 v1 = __ldg(reinterpret_cast<const double2 *>(brow + k + 2));
      const double2 w0 = __ldg(reinterpret_cast<const double2 *>(wv + k));
      const double2 w1 = __ldg(reinterpret_cast<const double2 *>(wv + k + 2));
      rb[0] = v0.x * w0.x; rb[1] = v0.y * w0.y; rb[2] = v1.x * w1.x; rb[3] = v1.y * w1.y;
    } else {
      rb[0] = rb[1] = rb[2] = rb[3] = 0.0;
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      sm.a[buf][lk + q][lr] = ra[q];
      sm.b[buf][lk + q][lr] = rb[q];
    }
  };
  if (k_begin < k_end) {
    gload(k_begin);
    sstore(0);
  }
  __syncthreads();
  int buf = 0;
  for (int k0 = k_begin; k0 < k_end; k0 += BK) {
    const bool more = k0 + BK < k_end;
    if (more) gload(k0 + BK);
    mma_slice(sm.a[buf], sm.b[buf], tx, ty, acc);
    if (more) sstore(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
  const int ntile = nblk * (nblk + 1) / 2;
  double *out = work + ((long)blockIdx.y * ntile + blockIdx.x) * (BM * BN);
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) out[row_of(ty, i) * BN + row_of(tx, j)] = acc[i][j];
}

__global__ void quadrature_reduce_kernel(int n, int nblk, int nchunk,
                                         const double *__restrict__ work,
                                         double *__restrict__ F) {
  const int ntile = nblk * (nblk + 1) / 2;
  const long total = (long)ntile * BM * BN;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const int tile = (int)(e / (BM * BN));
    const int m = (int)(e % (BM * BN)) / BN, c = (int)(e % BN);
    int mb = 0, rem = tile;
    while (rem >= nblk - mb) {
      rem -= nblk - mb;
      ++mb;
    }
    const int nb = mb + rem;
    const int mu = mb * BM + m, nu = nb * BN + c;
    if (mu >= n || nu >= n || mu > nu) continue;
    double s = 0.0;
    for (int k = 0; k < nchunk; ++k) s += work[((long)k * ntile + tile) * (BM * BN) + m * BN + c];
    F[(long)mu * n + nu] = s;
    F[(long)nu * n + mu] = s;
  }
}

__global__ void combine_weights_kernel(int npoint, const double *__restrict__ wb,
                                       const double *__restrict__ w, double q,
                                       const double *__restrict__ v,
                                       const double *__restrict__ vext,
                                       double *__restrict__ wv) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  double pot = v ? q * v[p] : 0.0;
  if (vext) pot += vext[p];
  wv[p] = wb[p] * w[p] * pot;
}

inline int quad_chunks(int n, int npoint_pad, int *chunk_out) {
  const int nblk = (n + BM - 1) / BM;
  const int ntile = nblk * (nblk + 1) / 2;
  // one CTA per SM at these register counts: aim for ~4 full waves over the
  // 148 SMs so the last wave is (nearly) full
  int nchunk = (4 * 148) / ntile;
  if (nchunk < 1) nchunk = 1;
  int chunk = (npoint_pad + nchunk - 1) / nchunk;
  chunk = ((chunk + BK - 1) / BK) * BK;
  if (chunk < BK) chunk = BK;
  nchunk = (npoint_pad + chunk - 1) / chunk;
  *chunk_out = chunk;
  return nchunk;
}

inline int pad_points(int npoint) { return ((npoint + BN - 1) / BN) * BN; }

}  // namespace

size_t density_workspace_bytes(int, int) { return 0; }

cudaError_t launch_density_f64(int n, int npoint, const double *phi, long ld,
                               const double *D, double *rho, cudaStream_t s) {
  if (npoint <= 0) return cudaSuccess;
  const int blocks = (npoint + BN - 1) / BN;
  density_kernel<<<blocks, NT, 0, s>>>(n, npoint, phi, ld, D, rho);
  return cudaGetLastError();
}

size_t quadrature_workspace_bytes(int n, int npoint) {
  int chunk;
  const int nchunk = quad_chunks(n, pad_points(npoint), &chunk);
  const int nblk = (n + BM - 1) / BM;
  return (size_t)nchunk * (nblk * (nblk + 1) / 2) * BM * BN * sizeof(double);
}

cudaError_t launch_quadrature_f64(int n, int npoint, const double *phi, long ld,
                                  const double *wv, double *F, double *work,
                                  cudaStream_t s, const double *phib) {
  if (!phib) phib = phi;
  if (n <= 0) return cudaSuccess;
  const int npad = pad_points(npoint);
  int chunk;
  const int nchunk = quad_chunks(n, npad, &chunk);
  const int nblk = (n + BM - 1) / BM;
  const int ntile = nblk * (nblk + 1) / 2;
  dim3 grid(ntile, nchunk);
  quadrature_kernel<<<grid, NT, 0, s>>>(n, npad, phi, phib, ld, wv, nblk, chunk, work);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long total = (long)ntile * BM * BN;
  const int rblocks = (int)std::min<long>((total + 255) / 256, 148 * 16);
  quadrature_reduce_kernel<<<rblocks, 256, 0, s>>>(n, nblk, nchunk, work, F);
  return cudaGetLastError();
}

cudaError_t launch_quadrature_reduce(int n, int nchunk, const double *work, double *F,
                                     cudaStream_t s) {
  const int nblk = (n + BM - 1) / BM;
  const int ntile = nblk * (nblk + 1) / 2;
  const long total = (long)ntile * BM * BN;
  const int rblocks = (int)std::min<long>((total + 255) / 256, 148 * 16);
  quadrature_reduce_kernel<<<rblocks, 256, 0, s>>>(n, nblk, nchunk, work, F);
  return cudaGetLastError();
}

cudaError_t launch_combine_weights(int npoint, const double *wb, const double *w,
                                   double q, const double *v, const double *vext,
                                   double *wv, cudaStream_t s) {
  if (npoint <= 0) return cudaSuccess;
  combine_weights_kernel<<<(npoint + 255) / 256, 256, 0, s>>>(npoint, wb, w, q, v,
                                                             vext, wv);
  return cudaGetLastError();
}

}  // namespace napmo

// ===========================================================================
// Allocation-free quadrature: napmo_gpu_quadrature_noalloc.
//
// Some callers of this library cannot allocate device memory while they call
// it: host applications that reserve and budget the whole memory of a GPU at
// start-up and hand plugins no allocator (a cudaMalloc from the plugin would
// take memory the host has already promised elsewhere, or fail), and callers
// that must not let an allocation stall or synchronise the device in the
// middle of their own work.  For them this entry point runs the same split-K
// quadrature kernels as napmo_gpu_quadrature, with the per-chunk partial tiles
// kept in `g_quad_scratch`, a fixed 16 MiB array compiled into the library:
// every GPU that loads libnapmo holds it until the process exits.
//
// Limit: the partial tiles of one chunk must fit, so n <= 1920 basis
// functions; larger n is rejected with an error before anything is launched.
// The chunk count is lowered to fit the array (fewer, longer chunks), so the
// result can differ from napmo_gpu_quadrature in the last bits (different
// summation grouping); it is deterministic from call to call.
//
// Address: every call looks up the device address of the array with
// cudaGetSymbolAddress, with the caller's device current, and passes it to the
// kernels (in host code the array's name is only a host-side stand-in).  The
// lookup allocates nothing; doing it per call rather than caching it keeps the
// address right under any context and after a device reset.  The first call
// on a device may load the library's device code there: make it before any
// stream capture.
//
// Inputs: phi, psi and wv are read with 16-byte loads up to npoint rounded up
// to 128, so they must be 16-byte aligned, ld even, and wv zero padded to that
// length (napmo_gpu_combine_weights writes it so).  npoint = 0 gives F = 0.
//
// Sharing: the array is shared by all calls and keeps the previous call's
// contents; nothing in it needs to start at zero (each chunk overwrites its
// own tiles before they are added).  Calls that overlap on the GPU (different
// streams, or different host threads without ordering) race on the array and
// must be serialised by the caller.
// ===========================================================================
namespace napmo {
namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(2) << 20;  // 16 MiB
__device__ __align__(256) double g_quad_scratch[kNoAllocScratchDoubles];

// Device address of g_quad_scratch in the current context.
int scratch_address(double **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_quad_scratch);
  if (e != cudaSuccess)
    return set_error(kCudaError, std::string("cudaGetSymbolAddress(quadrature scratch): ") +
                                     cudaGetErrorString(e));
  *out = static_cast<double *>(p);
  return kOk;
}

}  // namespace
}  // namespace napmo

extern "C" {

// F[mu][nu] = sum_p phi[mu][p] wv[p] psi[nu][p] (psi = phi when null), upper
// triangle mirrored, like napmo_gpu_quadrature, without allocating: the
// split-K scratch lives in a fixed 16 MiB device array (n <= 1920).  See the
// block comment above for the address lookup, the input contract and the
// sharing rules.
int napmo_gpu_quadrature_noalloc(int n, int npoint, const double *phi, const double *psi,
                                 long ld, const double *wv, double *F, void *stream) {
  using namespace napmo;
  clear_error();
  if (n <= 0 || npoint < 0) return set_error(kInvalidArgument, "n must be positive, npoint >= 0");
  const int npad = pad_points(npoint);
  if (ld < npad || ld % 2 != 0)
    return set_error(kInvalidArgument, "ld must be even and >= npoint rounded up to 128");
  const int nblk = (n + BM - 1) / BM;
  const int ntile = nblk * (nblk + 1) / 2;
  const size_t per_chunk = (size_t)ntile * BM * BN;
  if (per_chunk > kNoAllocScratchDoubles)
    return set_error(kInvalidArgument,
                     "napmo_gpu_quadrature_noalloc: n = " + std::to_string(n) +
                         " exceeds the 16 MiB fixed scratch (at most 1920 basis functions)");
  cudaStream_t s = (cudaStream_t)stream;
  if (npoint == 0) {  // empty grid: F = 0 (a memset allocates nothing)
    const cudaError_t e = cudaMemsetAsync(F, 0, (size_t)n * n * sizeof(double), s);
    if (e != cudaSuccess) return set_error(kCudaError, std::string("memset F: ") + cudaGetErrorString(e));
    return kOk;
  }
  double *scratch = nullptr;
  int st = scratch_address(&scratch);
  if (st != kOk) return st;
  // as many chunks as the launch policy wants, capped by the fixed array
  int chunk;
  int nchunk = quad_chunks(n, npad, &chunk);
  const int cap = (int)(kNoAllocScratchDoubles / per_chunk);
  if (nchunk > cap) {
    chunk = (npad + cap - 1) / cap;
    chunk = ((chunk + BK - 1) / BK) * BK;
    nchunk = (npad + chunk - 1) / chunk;
  }
  dim3 grid(ntile, nchunk);
  quadrature_kernel<<<grid, NT, 0, s>>>(n, npad, phi, psi ? psi : phi, ld, wv, nblk, chunk,
                                        scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(kCudaError, std::string("quadrature: ") + cudaGetErrorString(e));
  const long total = (long)ntile * BM * BN;
  const int rblocks = (int)std::min<long>((total + 255) / 256, 148 * 16);
  quadrature_reduce_kernel<<<rblocks, 256, 0, s>>>(n, nblk, nchunk, scratch, F);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(kCudaError, std::string("quadrature reduce: ") + cudaGetErrorString(e));
  return kOk;
}

}  // extern "C"
