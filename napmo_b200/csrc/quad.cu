// FP64 grid quadratures (the plain FP64 path) on the FP64 tensor pipe:
//
//   density     rho[p]     = sum_{mu,nu} phi[mu][p] D[mu][nu] phi[nu][p]
//   quadrature  F[mu][nu]  = sum_p phi[mu][p] wv[p] phi[nu][p]
//               (or sum_p phi[mu][p] wv[p] psi[nu][p] for a second operand psi,
//               upper triangle mirrored as nAPMO does for exchange)
//
// nAPMO computes the density point by point in Python (psi_hybrid.py:144-150)
// and the quadrature by materialising every orbital product
// Psi[n(n+1)/2][N] (src/wavefunction/nwavefunction.cpp:77-107,161-197).  Here
// both are FP64 GEMMs over phi stored basis-major [n][ld] (ld a multiple of
// 128, zero padded), issued as mma.sync m16n8k8 f64 (DMMA: 2048 flops per
// warp instruction, FP64 accumulation) from operand tiles that cp.async
// streams into a 4-stage shared-memory ring:
//
//   * density: a CTA owns 128 points and sweeps 128-row blocks of mu.  D is
//     folded onto block-upper-triangular form (block b of mu takes nu from
//     its own first row on; entries right of the diagonal block count twice,
//     exact for symmetric D), so the CTA forms T' = D' phi for each block
//     (62 % of the full product at n = 510) and folds T' into the per-point
//     sum with phi[mu][p] in the epilogue; deterministic, no atomics.
//   * quadrature: split-K over points.  CTA (tile, chunk) accumulates one
//     128x128 upper-triangle tile of F over one chunk of points into a
//     workspace slot (wv applied to the B fragments in registers); a second
//     kernel adds the chunks in fixed order and writes both triangles, so F
//     is exactly symmetric and bit-reproducible.
//
// Tiles: 128x128 per CTA, 8 warps as 2 x 4 of 64x32 (4 x 4 m16n8 tiles, 64
// FP64 accumulators per thread), 16 points (quadrature) or 16 functions
// (density) per stage.  Shared-memory rows are padded to a stride of 4 mod 16
// doubles, so the fragment loads of each half-warp hit 16 distinct banks.
#include <cstdint>
#include <string>

#include "common.h"
#include "dmma.cuh"
#include "kernels.cuh"

namespace napmo {

namespace {

constexpr int BM = 128, BN = 128, NT = 256;
constexpr int BK = 16;                 // points (quadrature) / functions (density) per stage
constexpr int NS = 4;                  // stages of the cp.async ring
constexpr int LDA = BK + 4;            // [row][k] tiles: stride 20 doubles
constexpr int LDB = BN + 4;            // density phi tile [nu][p]: stride 132 doubles

struct QuadSmem {
  double a[NS][BM][LDA];               // phi rows mu0.. over the stage's points
  double b[NS][BN][LDA];               // psi rows nu0..
  double w[NS][BK];                    // wv over the stage's points
};

struct DensSmem {
  double a[NS][BM][LDA];               // D' rows mu0.. over the stage's nu
  double b[NS][BK][LDB];               // phi rows nu over the CTA's 128 points
  double red[2][BN];                   // per-point sums of the two warp rows
};

constexpr size_t kQuadSmem = sizeof(QuadSmem);
constexpr size_t kDensSmem = sizeof(DensSmem);

// 16-byte / 8-byte asynchronous global -> shared copies; src_bytes = 0 fills
// the destination with zeros (rows beyond n) without reading the source.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
               "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
               "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// acc[mt][nt] += A-tile rows (warp rows mt) x B-tile columns (warp columns nt)
// over one stage: A fragments from a[row][k], B fragments from bf(col, k).
template <typename BFrag>
__device__ __forceinline__ void stage_mma(const double (*a)[LDA], int wrow, int g, int q,
                                          BFrag bf, double (&acc)[4][4][4]) {
#pragma unroll
  for (int kk = 0; kk < BK; kk += 8) {
    double b[4][2];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) bf(nt, kk, b[nt]);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      const int r = wrow + mt * 16 + g;
      const double af[4] = {a[r][kk + q], a[r + 8][kk + q], a[r][kk + q + 4],
                            a[r + 8][kk + q + 4]};
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], af, b[nt]);
    }
  }
}

// ------------------------------------------------------------------ density
// Stages of a CTA: block mb of mu takes nu from mb*BM to n (rounded up to BK),
// the blocks one after the other; within a block the nu right of the
// diagonal block come first and the diagonal block's own nu last, so the
// doubling of the off-diagonal part is one multiply of the accumulators
// before the first diagonal stage.  Returns k0 of stage `it` and sets its
// block, whether it is the block's first diagonal stage, and whether it is
// the block's last stage.
__device__ __forceinline__ int density_stage(int it, int nblk, int nk, int &mb, bool &first_diag,
                                             bool &last) {
  constexpr int SB = BM / BK;                   // stages per 128 functions
  mb = 0;
  int left = it;
  while (mb < nblk) {
    const int cnt = nk - mb * SB;
    if (left < cnt) break;
    left -= cnt;
    ++mb;
  }
  const int ndiag = min(SB, nk - mb * SB);      // diagonal-block stages
  const int noff = nk - mb * SB - ndiag;        // stages right of it
  last = left == noff + ndiag - 1;
  first_diag = left == noff;
  return left < noff ? ((mb + 1) * SB + left) * BK : (mb * SB + left - noff) * BK;
}

// groups (optional): the 128-point groups to compute (screened plans; the
// others hold no kept point); keep (optional): rho = 0 at dropped points.
// rho of the 128 points p0 .. p0 + 127 (one CTA; see density_kernel).
template <bool kVecD>
__device__ __forceinline__ void density_block(DensSmem &sm, int n, int npoint,
                                              const double *__restrict__ phi, long ld,
                                              const double *__restrict__ D,
                                              double *__restrict__ rho, int p0,
                                              const int *__restrict__ keep) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int wrow = (warp >> 2) * 64, wcol = (warp & 3) * 32;
  const int nblk = (n + BM - 1) / BM;
  const int nk = (n + BK - 1) / BK;                 // stages of nu over the whole basis
  int nstage = 0;
  for (int mb = 0; mb < nblk; ++mb) nstage += nk - mb * (BM / BK);

  // copies of one stage: D' rows (16-byte copies when n is even and D is
  // 16-byte aligned, else 8-byte) and phi rows (16-byte copies; p0 + c is
  // even, ld even)
  auto load_stage = [&](int it) {
    int mb;
    bool fd, ls;
    const int k0 = density_stage(it, nblk, nk, mb, fd, ls);
    const int slot = it % NS;
    if (kVecD) {
#pragma unroll
      for (int i = 0; i < (BM * BK / 2) / NT; ++i) {
        const int e = t + NT * i, r = e / (BK / 2), c = (e % (BK / 2)) * 2;
        const int mu = mb * BM + r, nu = k0 + c;
        const bool v = mu < n && nu < n;   // n even: nu + 1 < n as well
        cp_async16(&sm.a[slot][r][c], D + (v ? (long)mu * n + nu : 0), v);
      }
    } else {
#pragma unroll
      for (int i = 0; i < (BM * BK) / NT; ++i) {
        const int e = t + NT * i, r = e / BK, c = e % BK;
        const int mu = mb * BM + r, nu = k0 + c;
        const bool v = mu < n && nu < n;
        cp_async8(&sm.a[slot][r][c], D + (v ? (long)mu * n + nu : 0), v);
      }
    }
#pragma unroll
    for (int i = 0; i < (BK * BN / 2) / NT; ++i) {
      const int e = t + NT * i, r = e / (BN / 2), c = (e % (BN / 2)) * 2;
      const int nu = k0 + r;
      const bool v = nu < n;
      cp_async16(&sm.b[slot][r][c], phi + (v ? (long)nu * ld + p0 + c : 0), v);
    }
  };

  double part[4][2];
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) part[nt][0] = part[nt][1] = 0.0;
  double acc[4][4][4];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[mt][nt][i] = 0.0;

#pragma unroll
  for (int i = 0; i < NS - 1; ++i) {
    if (i < nstage) load_stage(i);
    cp_async_commit();
  }
  for (int it = 0; it < nstage; ++it) {
    cp_async_wait<NS - 2>();
    __syncthreads();
    if (it + NS - 1 < nstage) load_stage(it + NS - 1);
    cp_async_commit();
    int mb;
    bool first_diag, last;
    density_stage(it, nblk, nk, mb, first_diag, last);
    const int slot = it % NS;
    if (first_diag) {
      // the part right of the diagonal block counts twice (D symmetric)
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[mt][nt][i] *= 2.0;
    }
    const double(*bt)[LDB] = sm.b[slot];
    stage_mma(sm.a[slot], wrow, g, q,
              [&](int nt, int kk, double(&b)[2]) {
                const int c = wcol + nt * 8 + g;
                b[0] = bt[kk + q][c];
                b[1] = bt[kk + q + 4][c];
              },
              acc);
    // last stage of block mb: part[p] += sum_mu T'[mu][p] phi[mu][p]
    if (last) {
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int mu = mb * BM + wrow + mt * 16 + g + 8 * h;
          if (mu < n) {
            const double *prow = phi + (long)mu * ld + p0 + wcol + 2 * q;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
              const double2 f = __ldg(reinterpret_cast<const double2 *>(prow + nt * 8));
              part[nt][0] = fma(acc[mt][nt][2 * h], f.x, part[nt][0]);
              part[nt][1] = fma(acc[mt][nt][2 * h + 1], f.y, part[nt][1]);
            }
          }
        }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[mt][nt][i] = 0.0;
    }
  }
  cp_async_wait<0>();
  // sum over the warp's rows (lanes of equal q), then over the two warp rows
#pragma unroll
  for (int nt = 0; nt < 4; ++nt)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double v = part[nt][j];
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 8);
      v += __shfl_xor_sync(0xffffffffu, v, 16);
      part[nt][j] = v;
    }
  if (g == 0) {
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      sm.red[warp >> 2][wcol + nt * 8 + 2 * q] = part[nt][0];
      sm.red[warp >> 2][wcol + nt * 8 + 2 * q + 1] = part[nt][1];
    }
  }
  __syncthreads();
  if (t < BN && p0 + t < npoint)
    rho[p0 + t] = (keep && !keep[p0 + t]) ? 0.0 : sm.red[0][t] + sm.red[1][t];
}

template <bool kVecD>
__global__ void __launch_bounds__(NT, 1)
density_kernel(int n, int npoint, const double *__restrict__ phi, long ld,
               const double *__restrict__ D, double *__restrict__ rho,
               const int *__restrict__ groups, const int *__restrict__ keep) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  DensSmem &sm = *reinterpret_cast<DensSmem *>(smem_raw);
  const int p0 = (groups ? groups[blockIdx.x] : (int)blockIdx.x) * BN;
  density_block<kVecD>(sm, n, npoint, phi, ld, D, rho, p0, keep);
}

// --------------------------------------------------------------- quadrature
// Without `blocks` the K range is every point (npoint_pad, chunks of `chunk`
// points); with it (screened plans) the K range is the list of 16-point
// blocks holding a kept point, npoint_pad = 16 x their count and `chunk` a
// multiple of 16 as before.
// Tile `tile` (upper-triangle index) of F over chunk `ck` of the points into
// its workspace slot (one CTA; see quadrature_kernel).
__device__ __forceinline__ void quadrature_block(QuadSmem &sm, int n, int npoint_pad,
                                                 const double *__restrict__ phi,
                                                 const double *__restrict__ phib, long ld,
                                                 const double *__restrict__ wv, int nblk,
                                                 int chunk, double *__restrict__ work,
                                                 const int *__restrict__ blocks, int tile_index,
                                                 int ck) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int wrow = (warp >> 2) * 64, wcol = (warp & 3) * 32;
  // upper-triangle tile index -> (mb, nb)
  int tile = tile_index, mb = 0;
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
  const int k_begin = ck * chunk;
  const int k_end = min(k_begin + chunk, npoint_pad);
  const int nstage = k_end > k_begin ? (k_end - k_begin) / BK : 0;

  // copies of one stage: 128 rows x 16 points of each operand (8 x 16 bytes
  // per row) and the 16 weights; rows beyond n are zero filled
  auto load_stage = [&](int it) {
    const int kv = k_begin + it * BK;
    const int slot = it % NS, k0 = blocks ? blocks[kv / BK] * BK : kv;
#pragma unroll
    for (int i = 0; i < (BM * BK / 2) / NT; ++i) {
      const int e = t + NT * i, r = e / (BK / 2), c = (e % (BK / 2)) * 2;
      const bool va = mu0 + r < n, vb = nu0 + r < n;
      cp_async16(&sm.a[slot][r][c], phi + (va ? (long)(mu0 + r) * ld + k0 + c : 0), va);
      cp_async16(&sm.b[slot][r][c], phib + (vb ? (long)(nu0 + r) * ld + k0 + c : 0), vb);
    }
    if (t < BK / 2) cp_async16(&sm.w[slot][2 * t], wv + k0 + 2 * t, true);
  };

  double acc[4][4][4];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[mt][nt][i] = 0.0;

#pragma unroll
  for (int i = 0; i < NS - 1; ++i) {
    if (i < nstage) load_stage(i);
    cp_async_commit();
  }
  for (int it = 0; it < nstage; ++it) {
    cp_async_wait<NS - 2>();
    __syncthreads();
    if (it + NS - 1 < nstage) load_stage(it + NS - 1);
    cp_async_commit();
    const int slot = it % NS;
    const double(*bt)[LDA] = sm.b[slot];
    const double *w = sm.w[slot];
    stage_mma(sm.a[slot], wrow, g, q,
              [&](int nt, int kk, double(&b)[2]) {
                const int c = wcol + nt * 8 + g;
                b[0] = bt[c][kk + q] * w[kk + q];
                b[1] = bt[c][kk + q + 4] * w[kk + q + 4];
              },
              acc);
  }
  cp_async_wait<0>();
  const int ntile = nblk * (nblk + 1) / 2;
  double *out = work + ((long)ck * ntile + tile_index) * (BM * BN);
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int r = wrow + mt * 16 + g, c = wcol + nt * 8 + 2 * q;
      *reinterpret_cast<double2 *>(out + r * BN + c) = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
      *reinterpret_cast<double2 *>(out + (r + 8) * BN + c) =
          make_double2(acc[mt][nt][2], acc[mt][nt][3]);
    }
}

__global__ void __launch_bounds__(NT, 1)
quadrature_kernel(int n, int npoint_pad, const double *__restrict__ phi,
                  const double *__restrict__ phib, long ld,
                  const double *__restrict__ wv, int nblk, int chunk,
                  double *__restrict__ work, const int *__restrict__ blocks) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  QuadSmem &sm = *reinterpret_cast<QuadSmem *>(smem_raw);
  quadrature_block(sm, n, npoint_pad, phi, phib, ld, wv, nblk, chunk, work, blocks,
                   blockIdx.x, blockIdx.y);
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
                               const double *D, double *rho, cudaStream_t s,
                               const int *groups, int ngroup, const int *keep) {
  if (npoint <= 0) return cudaSuccess;
  int blocks = (npoint + BN - 1) / BN;
  if (groups) {
    // groups without a kept point are not computed: their rho is 0
    cudaError_t e = cudaMemsetAsync(rho, 0, (size_t)npoint * sizeof(double), s);
    if (e != cudaSuccess) return e;
    blocks = ngroup;
    if (blocks == 0) return cudaSuccess;
  }
  // 16-byte copies of D rows need n even and a 16-byte aligned D
  const bool vec = n % 2 == 0 && reinterpret_cast<uintptr_t>(D) % 16 == 0;
  auto kern = vec ? density_kernel<true> : density_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kDensSmem);
  if (e != cudaSuccess) return e;
  kern<<<blocks, NT, kDensSmem, s>>>(n, npoint, phi, ld, D, rho, groups, keep);
  return cudaGetLastError();
}

// the split-K quadrature kernel with its dynamic shared memory
cudaError_t quadrature_launch(dim3 grid, int n, int npad, const double *phi, const double *phib,
                              long ld, const double *wv, int nblk, int chunk, double *work,
                              cudaStream_t s, const int *blocks = nullptr) {
  cudaError_t e = cudaFuncSetAttribute(quadrature_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kQuadSmem);
  if (e != cudaSuccess) return e;
  quadrature_kernel<<<grid, NT, kQuadSmem, s>>>(n, npad, phi, phib, ld, wv, nblk, chunk, work,
                                                blocks);
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
                                  cudaStream_t s, const double *phib, const int *blocks,
                                  int nblock) {
  if (!phib) phib = phi;
  if (n <= 0) return cudaSuccess;
  // screened: the K range is the listed 16-point blocks; its chunk count is
  // capped at the workspace's (sized for every point), see quadrature_chunking
  const int npad = blocks ? nblock * BK : pad_points(npoint);
  if (npad == 0) return cudaMemsetAsync(F, 0, (size_t)n * n * sizeof(double), s);
  int chunk;
  const int nchunk = quadrature_chunking(n, npad, &chunk, pad_points(npoint));
  const int nblk = (n + BM - 1) / BM;
  const int ntile = nblk * (nblk + 1) / 2;
  dim3 grid(ntile, nchunk);
  cudaError_t e = quadrature_launch(grid, n, npad, phi, phib, ld, wv, nblk, chunk, work, s,
                                    blocks);
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

// -------------------------------------------------------------- batches
// Persistent batched launches: CTAs take (molecule, tile) items from a device
// work queue until it is empty.  Item i may be taken once *posted > i (the
// batch posts its items when it is built; a producer that never posts makes
// the wait run out): the wait is bounded by q.timeout_ns of %globaltimer,
// after which the CTA records kDeviceTimeout in *q.status and stops.
namespace {

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ int queue_pop(const BatchQueue &q) {
  const int i = atomicAdd(q.head, 1);
  if (i >= q.nitems) return -1;
  const volatile int *posted = q.posted;
  if (*posted > i) return i;
  const unsigned long long t0 = globaltimer_ns();
  for (unsigned it = 1;; ++it) {
    if (*posted > i) return i;
    if ((it & 63) == 0 && globaltimer_ns() - t0 > q.timeout_ns) {
      atomicExch(q.status, kDeviceTimeout);
      return -1;
    }
  }
}

// the CTA's next item (all threads), -1 when the queue is done
__device__ __forceinline__ int cta_pop(const BatchQueue &q, int *slot) {
  if (threadIdx.x == 0) *slot = queue_pop(q);
  __syncthreads();
  const int w = *slot;
  __syncthreads();
  return w;
}

__global__ void __launch_bounds__(NT, 1)
density_batch_kernel(const DensBatchArg *__restrict__ args, BatchQueue q) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  DensSmem &sm = *reinterpret_cast<DensSmem *>(smem_raw);
  __shared__ int slot;
  for (;;) {
    const int w = cta_pop(q, &slot);
    if (w < 0) break;
    const int4 it = q.items[w];
    const DensBatchArg a = args[it.x];
    if (a.vecD)
      density_block<true>(sm, a.n, a.npoint, a.phi, a.ld, a.D, a.rho, it.y * BN, a.keep);
    else
      density_block<false>(sm, a.n, a.npoint, a.phi, a.ld, a.D, a.rho, it.y * BN, a.keep);
  }
}

__global__ void __launch_bounds__(NT, 1)
quadrature_batch_kernel(const QuadBatchArg *__restrict__ args, BatchQueue q) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  QuadSmem &sm = *reinterpret_cast<QuadSmem *>(smem_raw);
  __shared__ int slot;
  for (;;) {
    const int w = cta_pop(q, &slot);
    if (w < 0) break;
    const int4 it = q.items[w];
    const QuadBatchArg a = args[it.x];
    quadrature_block(sm, a.n, a.npad, a.phi, a.phi, a.ld, a.wv, a.nblk, a.chunk, a.work,
                     a.blocks, it.y, it.z);
  }
}

// F of every molecule from its chunk partials (blockIdx.y = molecule)
__global__ void quadrature_reduce_batch_kernel(const QuadBatchArg *__restrict__ args) {
  const QuadBatchArg a = args[blockIdx.y];
  const int ntile = a.nblk * (a.nblk + 1) / 2;
  const long total = (long)ntile * BM * BN;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const int tile = (int)(e / (BM * BN));
    const int m = (int)(e % (BM * BN)) / BN, c = (int)(e % BN);
    int mb = 0, rem = tile;
    while (rem >= a.nblk - mb) {
      rem -= a.nblk - mb;
      ++mb;
    }
    const int nb = mb + rem;
    const int mu = mb * BM + m, nu = nb * BN + c;
    if (mu >= a.n || nu >= a.n || mu > nu) continue;
    double s = 0.0;
    for (int k = 0; k < a.nchunk; ++k) s += a.work[((long)k * ntile + tile) * (BM * BN) + m * BN + c];
    a.F[(long)mu * a.n + nu] = s;
    a.F[(long)nu * a.n + mu] = s;
  }
}

// wv of every molecule (blockIdx.y), zero padded to its npad points
__global__ void combine_weights_batch_kernel(const WeightBatchArg *__restrict__ args, double q) {
  const WeightBatchArg a = args[blockIdx.y];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.npad; p += gridDim.x * blockDim.x)
    a.wv[p] = p < a.npoint ? a.wb[p] * a.w[p] * (q * a.v[p]) : 0.0;
}

}  // namespace

// Chunking of a K range of npad points when the workspace was sized for a
// grid of pad_full points (npad <= pad_full): quad_chunks is not monotone in
// the range (a shorter range below a chunk-size step gets more, shorter
// chunks), so the chunk count is capped at the full grid's and the chunks
// lengthened to fit.
int quadrature_chunking(int n, int npad, int *chunk, int pad_full) {
  int c = 0;
  int nchunk = quad_chunks(n, npad, &c);
  int cf = 0;
  const int cap = quad_chunks(n, pad_full > npad ? pad_full : npad, &cf);
  if (nchunk > cap) {
    c = (npad + cap - 1) / cap;
    c = ((c + BK - 1) / BK) * BK;
    nchunk = (npad + c - 1) / c;
  }
  *chunk = c;
  return nchunk;
}

cudaError_t launch_density_batch(const DensBatchArg *args, const BatchQueue &q, int grid,
                                 cudaStream_t s) {
  if (q.nitems == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(density_batch_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kDensSmem);
  if (e != cudaSuccess) return e;
  density_batch_kernel<<<grid, NT, kDensSmem, s>>>(args, q);
  return cudaGetLastError();
}

cudaError_t launch_quadrature_batch(const QuadBatchArg *args, const BatchQueue &q, int grid,
                                    cudaStream_t s) {
  if (q.nitems == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(quadrature_batch_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kQuadSmem);
  if (e != cudaSuccess) return e;
  quadrature_batch_kernel<<<grid, NT, kQuadSmem, s>>>(args, q);
  return cudaGetLastError();
}

cudaError_t launch_quadrature_reduce_batch(const QuadBatchArg *args, int nmol, cudaStream_t s) {
  if (nmol == 0) return cudaSuccess;
  quadrature_reduce_batch_kernel<<<dim3(148 * 2, nmol), 256, 0, s>>>(args);
  return cudaGetLastError();
}

cudaError_t launch_combine_weights_batch(const WeightBatchArg *args, int nmol, double q,
                                         cudaStream_t s) {
  if (nmol == 0) return cudaSuccess;
  combine_weights_batch_kernel<<<dim3(148, nmol), 256, 0, s>>>(args, q);
  return cudaGetLastError();
}

// ------------------------------------------------------ FP64 point screening
namespace {

// keep[p] = 1 when |wb w| max_mu phi_mu(p)^2 >= tol (the test of the int8
// plans: a dropped point changes an element of F by at most tol |v(p)|).
__global__ void screen_points_kernel(const double *__restrict__ phi, long ld, int n, int npoint,
                                     const double *__restrict__ wb, const double *__restrict__ w,
                                     double tol, int *__restrict__ keep) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  double mx = 0.0;
  for (int mu = 0; mu < n; ++mu) mx = fmax(mx, fabs(__ldg(phi + (long)mu * ld + p)));
  const double t = fabs(wb[p] * w[p]);
  keep[p] = (t * mx) * mx >= tol ? 1 : 0;
}

// flags[b] = 1 when block b of `span` points holds a kept point
__global__ void screen_blocks_kernel(const int *__restrict__ keep, int npoint, int span,
                                     int nb, int *__restrict__ flags) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int any = 0;
  for (int i = b * span; i < min((b + 1) * span, npoint); ++i) any |= keep[i];
  flags[b] = any;
}

}  // namespace

cudaError_t launch_fp64_screening(int n, int npoint, const double *phi, long ld, const double *wb,
                                  const double *w, double tol, int *keep, int *block_flags,
                                  int *group_flags, cudaStream_t s) {
  if (npoint <= 0) return cudaSuccess;
  screen_points_kernel<<<(npoint + 255) / 256, 256, 0, s>>>(phi, ld, n, npoint, wb, w, tol,
                                                           keep);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int nb = (npoint + BK - 1) / BK, ng = (npoint + BN - 1) / BN;
  screen_blocks_kernel<<<(nb + 255) / 256, 256, 0, s>>>(keep, npoint, BK, nb, block_flags);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  screen_blocks_kernel<<<(ng + 255) / 256, 256, 0, s>>>(keep, npoint, BN, ng, group_flags);
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
  cudaError_t e = quadrature_launch(grid, n, npad, phi, psi ? psi : phi, ld, wv, nblk, chunk,
                                    scratch, s);
  if (e != cudaSuccess) return set_error(kCudaError, std::string("quadrature: ") + cudaGetErrorString(e));
  const long total = (long)ntile * BM * BN;
  const int rblocks = (int)std::min<long>((total + 255) / 256, 148 * 16);
  quadrature_reduce_kernel<<<rblocks, 256, 0, s>>>(n, nblk, nchunk, scratch, F);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(kCudaError, std::string("quadrature reduce: ") + cudaGetErrorString(e));
  return kOk;
}

}  // extern "C"
