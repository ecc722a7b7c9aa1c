// Mixed-precision grid quadratures on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, int32 accumulators in TMEM), sm_100a.
//
//   quadrature  F[mu][nu] = sum_p phi[mu][p] wv[p] phi[nu][p]
//   density     rho[p]    = sum_mu phi[mu][p] (D phi)[mu][p]
//
// Slices.  The FP64 values of a group (one basis function over a block of 1024
// points; all basis functions at one point; one row of D) share the group
// exponent e (max |x| < 2^e).  Each value is rounded once, to the integer
// Y = rint(x 2^(30 - e)) (|Y| <= 2^30, error <= 2^-31 of the group maximum),
// and Y is written in balanced base 256 as four int8 digits
//   Y = d0 2^24 + d1 2^16 + d2 2^8 + d3,   |d0| <= 64, -128 <= dk <= 127.
// A product of two sliced operands keeps the digit products d_i d'_j with
// i + j <= 4.  The products of one diagonal i + j share an int32 TMEM
// accumulator, so the accumulation is exact: besides the slicing, the only
// error is the dropped digit products (relative 2^-37 of the group maxima).
// D (density) gets a fifth digit, Y = rint(x 2^(38 - e)): its rounding enters
// the energy through every element of D at once.  The drain
// combines the diagonals in int64, converts once to FP64 and applies the group
// exponents; FP64 partials are summed in a fixed order (deterministic).
//
// Quadrature weights span many decades across a block of points, so the
// weight is split between the operands by a power of two per point:
// A = phi 2^c(p), B = wv phi 2^-c(p), c(p) = floor(log2 |wb w| / 2) (exact).
//
// Operand images.  Each operand lives in HBM as tiles already in the
// no-swizzle K-major shared-memory layout of the tensor core (core matrices
// of 8 rows x 16 bytes; element (r, k) of a 64-wide K stage of one slice at
// (r / 8) * 512 + (k / 16) * 128 + (r % 8) * 16 + k % 16), the four slices of
// a stage contiguous, so one cp.async.bulk moves a stage of an operand.  phi's
// images are built once per grid; wv phi (quadrature) and D (density) are
// sliced on every call.
//
// Point screening.  A plan may keep only the points whose weight can matter:
// |wb w| max_mu phi_mu(p)^2 >= screen_tol.  Every term of the density's
// Poisson projection and of the quadrature carries wb w and a product of two
// basis functions at the point, so a dropped point changes F by at most
// screen_tol |v(p)| per matrix element.  The images then hold the kept points
// only (idx[k] = grid index of compacted point k); rho is scattered back and
// is 0 at dropped points.
//
// Kernels: warp 12 (one thread) streams stages into a 3-slot ring
// (cp.async.bulk + mbarrier transaction counts), warp 13 (one thread) issues
// the MMAs and owns TMEM, warps 0-11 drain TMEM.  Every mbarrier wait is
// bounded (2 s of globaltimer, or another role's abort): on timeout the kernel
// records an error in g_tc_error, the roles stop, copies and MMAs in flight
// are waited for (bounded) and TMEM is freed before the CTA exits.
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <atomic>
#include <cstdint>
#include <memory>

#include "capi_common.cuh"
#include "common.h"
#include "kernels.cuh"

namespace napmo {

__device__ int g_tc_error = 0;

namespace {

constexpr int KS = 64;            // K elements per stage = bytes per row of one slice
constexpr int NSL = 4;            // int8 slices per value
constexpr int NSL_D = 5;          // slices of D (density), 39 bits
constexpr int TM = 128;           // M tile (TMEM lanes)
constexpr int QN = 96;            // quadrature N tile: 5 diagonals x 96 columns
constexpr int DN = 96;            // density N tile: 5 diagonals x 96 columns
constexpr int QKB = 1024;         // quadrature exponent block (points)
constexpr int QBLK_STAGES = QKB / KS;
constexpr int NSTAGE = 3;
constexpr int kScaleWarps = 8;    // warps of a B-image CTA (2 stages each)
// Three drain warps per TMEM lane quadrant, 32 of the 96 columns each: the
// drain's per-column work waits on TMEM and global loads, and the MMAs of the
// next pass (or exponent block) wait for it.
constexpr int NEPI = 384;         // drain threads (warps 0-11)
constexpr int NTHR = NEPI + 64;   // + producer warp 12 + MMA warp 13
constexpr int kWarpP = NEPI / 32, kWarpM = NEPI / 32 + 1;  // producer, MMA warps
constexpr int DCW = 96 / (NEPI / 128);  // columns per drain warp
constexpr int kTmemCols = 512;
constexpr int kEmin = -960;
constexpr unsigned long long kTimeoutNs = 2000000000ull;

__host__ __device__ constexpr int stage_bytes(int rows) { return NSL * rows * KS; }

__host__ __device__ __forceinline__ int core_off(int r, int k) {
  return (r >> 3) * 512 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

// Digit products (i, j) with i + j <= 4 in diagonal order: (0,0) | (0,1) (1,0) |
// (0,2) (1,1) (2,0) | (0,3) (1,2) (2,1) (3,0) | then diagonal 4: for the
// quadrature (both operands 4 digits) (1,3) (2,2) (3,1), 13 products; for the
// density (B = D with 5 digits) (0,4) (1,3) (2,2) (3,1), 14 products.
constexpr int kQuadProducts = 13, kDensProducts = 14;
__host__ __device__ constexpr int prod_diag(int q) {
  return q < 1 ? 0 : q < 3 ? 1 : q < 6 ? 2 : q < 10 ? 3 : 4;
}
__host__ __device__ constexpr int prod_i(int q, bool b5) {
  return q < 10 ? q - prod_diag(q) * (prod_diag(q) + 1) / 2 : (b5 ? q - 10 : q - 9);
}
__host__ __device__ constexpr int prod_j(int q, bool b5) { return prod_diag(q) - prod_i(q, b5); }

// kind::i8 instruction descriptor: S32 accumulator, signed A and B, both
// K-major, N columns, M = 128.
constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(TM >> 4) << 24);
}

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void named_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// global -> shared bulk copy (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase of `bar` with parity `parity`.  Gives up when another
// role has set *abort, or after kTimeoutNs; a timeout records kDeviceTimeout
// and sets *abort.  abort == nullptr: only the time limit applies.
__device__ bool wait_phase(uint64_t *bar, uint32_t parity, volatile int *abort) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63) == 0) {
      if (abort && *abort) return false;
      if (global_ns() - t0 > kTimeoutNs) {
        if (abort) *abort = 1;
        atomicExch(&g_tc_error, kDeviceTimeout);
        return false;
      }
    }
  }
}

// The drain warps' wait: thread 0 polls, the outcome is shared through smem so
// that all nepi drain threads take the same branch.
__device__ bool group_wait(uint64_t *bar, uint32_t parity, volatile int *abort,
                           volatile int *flag, int nepi) {
  if (threadIdx.x == 0) *flag = wait_phase(bar, parity, abort) ? 1 : 0;
  named_sync(1, nepi);
  const bool ok = *flag != 0;
  named_sync(1, nepi);
  return ok;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  // no swizzle, K-major: LBO = 128 B (next 16 bytes of K), SBO = 512 B (next
  // 8 rows), descriptor version 1
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 8 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int32_t *v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// ties loaded registers to a point after the wait, so no use is scheduled
// before it
__device__ __forceinline__ void tie8(int32_t *v) {
  asm volatile("" : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
               "+r"(v[6]), "+r"(v[7]));
}

// ------------------------------------------------------------------ slices
__device__ __forceinline__ int group_exponent(double m) {
  if (!(m > 0.0)) return 0;
  int e;
  frexp(m, &e);
  return e < kEmin ? kEmin : e;
}

// 2^e as a double; 0 below the normal range (such terms are < 2^-960 of the
// results they enter).
__device__ __forceinline__ double pow2(int e) {
  return e < -1022 ? 0.0 : __longlong_as_double((long long)(e + 1023) << 52);
}

// Balanced base-256 digits by byte arithmetic.  For |Y| < 2^31 - 2^24, the
// balanced digits Y = d0 2^24 + d1 2^16 + d2 2^8 + d3 (-128 <= d1..d3 <= 127)
// are the bytes of U = Y + 0x808080: bytes 0..2 of U are d3 + 128, d2 + 128,
// d1 + 128 (no carries by construction) and byte 3 is d0.  So the int8 digit
// bytes (d & 255) of one element are the bytes of U ^ 0x808080, and the
// element is (W ^ 0x808080) - 0x808080 for its digit bytes W.  Four elements
// and four slices are a 4 x 4 byte transpose (8 byte permutations).
__device__ __forceinline__ void bytes_transpose4(uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                                 uint32_t *o) {
  // o[k] byte j = byte k of input j (inputs a, b, c, d = j 0..3)
  const uint32_t lo01 = __byte_perm(a, b, 0x5140), lo23 = __byte_perm(c, d, 0x5140);
  const uint32_t hi01 = __byte_perm(a, b, 0x7362), hi23 = __byte_perm(c, d, 0x7362);
  o[0] = __byte_perm(lo01, lo23, 0x5410);
  o[1] = __byte_perm(lo01, lo23, 0x7632);
  o[2] = __byte_perm(hi01, hi23, 0x5410);
  o[3] = __byte_perm(hi01, hi23, 0x7632);
}

// Four slices (d0 .. d3 words, byte e = element e) of four integers.
__device__ __forceinline__ void digits4(const int *y, uint32_t *w) {
  uint32_t t[4];
  bytes_transpose4(((uint32_t)y[0] + 0x808080u) ^ 0x808080u, ((uint32_t)y[1] + 0x808080u) ^ 0x808080u,
                   ((uint32_t)y[2] + 0x808080u) ^ 0x808080u, ((uint32_t)y[3] + 0x808080u) ^ 0x808080u,
                   t);
  // t[k] holds byte k of every element: k = 0 is d3 ... k = 3 is d0
  w[0] = t[3];
  w[1] = t[2];
  w[2] = t[1];
  w[3] = t[0];
}

// The four integers of four slice words (inverse of digits4).
__device__ __forceinline__ void undigits4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3,
                                          int *y) {
  uint32_t t[4];
  bytes_transpose4(w3, w2, w1, w0, t);  // t[e] bytes: d3, d2, d1, d0 of element e
#pragma unroll
  for (int e = 0; e < 4; ++e) y[e] = (int)(t[e] ^ 0x808080u) - 0x808080;
}

// Four balanced base-256 digit slices of rint(x[i] * scale), i < 16, packed
// one byte per element (slice s in out[s]).
__device__ __forceinline__ void slice16(const double *x, double scale, uint4 *out) {
  uint32_t w[4][4];  // [element group][slice]
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int y[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) y[e] = __double2int_rn(x[4 * q + e] * scale);
    digits4(y, w[q]);
  }
#pragma unroll
  for (int s = 0; s < NSL; ++s) out[s] = make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
}

// The 16 integers of four digit slices (inverse of slice16's packing).
__device__ __forceinline__ void unslice16(const uint4 *q, int *y) {
#pragma unroll
  for (int g = 0; g < 4; ++g)
    undigits4((&q[0].x)[g], (&q[1].x)[g], (&q[2].x)[g], (&q[3].x)[g], y + 4 * g);
}

// Five balanced base-256 digit slices of rint(x[i] * scale) (|.| <= 2^38;
// |d0| <= 64), packed one byte per element.
__device__ __forceinline__ void slice16_5(const double *x, double scale, uint4 *out) {
  uint32_t w[5][4];
#pragma unroll
  for (int s = 0; s < 5; ++s)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[s][q] = 0u;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    long long y = __double2ll_rn(x[i] * scale);
    int d[5];
#pragma unroll
    for (int k = 4; k > 0; --k) {
      d[k] = (int)(((y + 128) & 255) - 128);
      y = (y - d[k]) >> 8;
    }
    d[0] = (int)y;
    const int q = i >> 2, sh = (i & 3) * 8;
#pragma unroll
    for (int s = 0; s < 5; ++s) w[s][q] |= (uint32_t)(d[s] & 255) << sh;
  }
#pragma unroll
  for (int s = 0; s < 5; ++s) out[s] = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
}


// Row-grouped slices of X[row][k] = src[row * ld + k] * m1[k] * m2[k]
// (m1, m2 optional; X = 0 for row >= nrows or k >= ncols): exponent per
// (row, block of kb columns) in e[row * nblk + b]; image tiles of TR rows x KS
// columns, img[((row / TR) * nks + k / KS) * NSL * TR * KS + s * TR * KS +
// core_off(row % TR, k % KS)] with NS slices (4: Y = rint(x 2^(30-e)); 5:
// rint(x 2^(38-e))).  Grid (rows_pad / 8, nblk), one warp per row.
template <int NS>
__device__ __forceinline__ void slice_rows_body(const double *__restrict__ src, long ld,
                                                int nrows, int ncols,
                                                const double *__restrict__ m1,
                                                const double *__restrict__ m2, int kb, int nblk,
                                                int TR, int nks, int8_t *__restrict__ img,
                                                int *__restrict__ eout,
                                                const int *__restrict__ cidx, int bx, int by) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = bx * 8 + warp;
  const int b = by;
  const long k0 = (long)b * kb;
  const int nchunk = kb / 16;
  const bool vec = ((ld & 1) == 0);
  auto load = [&](int c, double *x) {
    const long k = k0 + (long)c * 16;
    if (row < nrows && k + 16 <= ncols) {
      const double *p = src + (long)row * ld + k;
      if (cidx) {  // column k is source column cidx[k]
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = __ldg(src + (long)row * ld + __ldg(cidx + k + i));
      } else if (vec) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const double2 v = __ldg(reinterpret_cast<const double2 *>(p) + q);
          x[2 * q] = v.x;
          x[2 * q + 1] = v.y;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = __ldg(p + i);
      }
      if (m1) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const double2 v = __ldg(reinterpret_cast<const double2 *>(m1 + k) + q);
          x[2 * q] *= v.x;
          x[2 * q + 1] *= v.y;
        }
      }
      if (m2) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const double2 v = __ldg(reinterpret_cast<const double2 *>(m2 + k) + q);
          x[2 * q] *= v.x;
          x[2 * q + 1] *= v.y;
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        double v = 0.0;
        if (row < nrows && k + i < ncols) {
          v = __ldg(src + (long)row * ld + (cidx ? __ldg(cidx + k + i) : k + i));
          if (m1) v *= __ldg(m1 + k + i);
          if (m2) v *= __ldg(m2 + k + i);
        }
        x[i] = v;
      }
    }
  };
  double mx = 0.0;
  for (int c = lane; c < nchunk; c += 32) {
    double x[16];
    load(c, x);
#pragma unroll
    for (int i = 0; i < 16; ++i) mx = fmax(mx, fabs(x[i]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const int e = group_exponent(mx);
  if (lane == 0) eout[(long)row * nblk + b] = e;
  const double scale = ldexp(1.0, 8 * NS - 2 - e);
  const int rt = row / TR, r = row % TR;
  const long tile = (long)NS * TR * KS;
  for (int c = lane; c < nchunk; c += 32) {
    double x[16];
    load(c, x);
    uint4 d[NS];
    if (NS == 5)
      slice16_5(x, scale, d);
    else
      slice16(x, scale, d);
    const long k = k0 + (long)c * 16;
    int8_t *base = img + ((long)rt * nks + k / KS) * tile + core_off(r, (int)(k % KS));
#pragma unroll
    for (int s = 0; s < NS; ++s)
      *reinterpret_cast<uint4 *>(base + (long)s * TR * KS) = d[s];
  }
}

template <int NS>
__global__ void __launch_bounds__(256)
slice_rows_kernel(const double *__restrict__ src, long ld, int nrows, int ncols,
                  const double *__restrict__ m1, const double *__restrict__ m2, int kb, int nblk,
                  int TR, int nks, int8_t *__restrict__ img, int *__restrict__ eout,
                  const int *__restrict__ cidx) {
  slice_rows_body<NS>(src, ld, nrows, ncols, m1, m2, kb, nblk, TR, nks, img, eout, cidx,
                      blockIdx.x, blockIdx.y);
}

// Point-grouped slices of phi^T: rows = points (tiles of 128), K = basis
// function (stages of 64); exponent per point over all n functions.  One
// thread per point, grid = padded points / 128.
__global__ void __launch_bounds__(TM)
slice_points_kernel(const double *__restrict__ phi, long ld, int n, int npoint, int nks,
                    int8_t *__restrict__ img, int *__restrict__ eout,
                    const int *__restrict__ pidx) {
  const int r = threadIdx.x;
  const long pk = (long)blockIdx.x * TM + r;
  const bool valid = pk < npoint;
  const long p = valid && pidx ? __ldg(pidx + pk) : pk;  // grid index of the point
  double mx = 0.0;
  if (valid)
    for (int nu = 0; nu < n; ++nu) mx = fmax(mx, fabs(__ldg(phi + (long)nu * ld + p)));
  const int e = group_exponent(mx);
  eout[pk] = e;
  const double scale = ldexp(1.0, 30 - e);
  const long tile = (long)NSL * TM * KS;
  for (int ks = 0; ks < nks; ++ks) {
#pragma unroll 1
    for (int kc = 0; kc < KS / 16; ++kc) {
      const int nu0 = ks * KS + kc * 16;
      double x[16];
#pragma unroll
      for (int i = 0; i < 16; ++i)
        x[i] = (valid && nu0 + i < n) ? __ldg(phi + (long)(nu0 + i) * ld + p) : 0.0;
      uint4 d[NSL];
      slice16(x, scale, d);
      int8_t *base = img + ((long)blockIdx.x * nks + ks) * tile + core_off(r, kc * 16);
#pragma unroll
      for (int s = 0; s < NSL; ++s) *reinterpret_cast<uint4 *>(base + (long)s * TM * KS) = d[s];
    }
  }
}

// sc[p] = 2^c(p), isc[p] = 2^-c(p), c(p) = floor(log2 |wb w| / 2) (0 where the
// weight is zero).  Some Lebedev rules have negative weights: the magnitude is
// split, the sign stays with wv.
__global__ void balance_kernel(int npoint, const double *__restrict__ wb,
                               const double *__restrict__ w, const int *__restrict__ pidx,
                               double *__restrict__ sc, double *__restrict__ isc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  const int q = pidx ? pidx[p] : p;
  const double t = fabs(wb[q] * w[q]);
  int c = 0;
  if (t > 0.0 && t < 1e300) {
    int ex;
    frexp(t, &ex);
    c = (ex - 1) >> 1;
    c = c < -400 ? -400 : (c > 400 ? 400 : c);
  }
  sc[p] = ldexp(1.0, c);
  isc[p] = ldexp(1.0, -c);
}

// Per call, block b of QKB points: g(p) = wv(p) isc(p)^2 (so that
// B = A g = phi wv 2^-c), eg[b] = group exponent of max |g| over the block,
// gs(p) = g(p) 2^-eg[b] (|gs| < 1; exact scaling).
__device__ __forceinline__ void gscale_body(int npoint, const double *__restrict__ wv,
                                            const double *__restrict__ isc,
                                            const int *__restrict__ pidx,
                                            double *__restrict__ gs, int *__restrict__ eg, int bx) {
  constexpr int PER = QKB / 256;
  __shared__ double red[8];
  const int t = threadIdx.x;
  const long p0 = (long)bx * QKB + t * PER;
  double g[PER], mx = 0.0;
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const long p = p0 + i;
    g[i] = p < npoint ? wv[pidx ? pidx[p] : p] * isc[p] * isc[p] : 0.0;
    mx = fmax(mx, fabs(g[i]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((t & 31) == 0) red[t >> 5] = mx;
  __syncthreads();
  mx = red[0];
#pragma unroll
  for (int i = 1; i < 8; ++i) mx = fmax(mx, red[i]);
  const int e = group_exponent(mx);
  if (t == 0) eg[bx] = e;
  const double s = ldexp(1.0, -e);
#pragma unroll
  for (int i = 0; i < PER; ++i) gs[p0 + i] = g[i] * s;
}

__global__ void __launch_bounds__(256)
gscale_kernel(int npoint, const double *__restrict__ wv, const double *__restrict__ isc,
              const int *__restrict__ pidx, double *__restrict__ gs, int *__restrict__ eg) {
  gscale_body(npoint, wv, isc, pidx, gs, eg, blockIdx.x);
}

// Per call: the B image from the A image.  For each row and block,
// x(p) = Y_A(p) gs(p) (|x| < 2^30); Y_B = rint(x 2^s) with s = 30 - e,
// e = group exponent of max |x| over the block, so B keeps 31 bits of its own
// block maximum; eb[b][row] = ea[row][b] + eg[b] - s (block-major, ebld rows
// per block, so a drain thread's columns are contiguous).  CTA = (8-row group,
// block), kScaleWarps warps; in every stage the row group's 8 rows x 64
// points of one slice are 512 contiguous bytes, so lane c holds the 16-byte
// chunk of row c & 7, points 16 (c >> 3) .. +15.  Warp w takes SPW stages from
// SPW w and keeps their Y_A, decoded once from the digits, in registers across
// both passes (row maxima: lanes c, c ^ 8, c ^ 16, c ^ 24, then the warps
// through shared memory; digits of B), so A is read from memory once.
__device__ __forceinline__ void scale_image_body(const int8_t *__restrict__ qa,
                                                 int8_t *__restrict__ qb,
                                                 const double *__restrict__ gs,
                                                 const int *__restrict__ ea,
                                                 const int *__restrict__ eg, int *__restrict__ eb,
                                                 int nks, int nblk, int ebld, int bx, int by) {
  constexpr int SPW = QBLK_STAGES / kScaleWarps;  // stages per warp
  __shared__ double smax[kScaleWarps][8];
  const int c = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rg = bx, b = by;
  const int t = rg >> 4, r = c & 7, kc = c >> 3;
  const int row = rg * 8 + r;
  const long goff = (long)(rg & 15) * 512 + c * 16;
  auto stage_base = [&](int st) {
    return ((long)t * nks + b * QBLK_STAGES + w * SPW + st) * stage_bytes(TM) + goff;
  };
  // Y_A of the thread's 64 elements, decoded once from the four digit slices
  int ya[SPW][16];
#pragma unroll
  for (int st = 0; st < SPW; ++st) {
    uint4 q[NSL];
#pragma unroll
    for (int s = 0; s < NSL; ++s)
      q[s] = __ldg(reinterpret_cast<const uint4 *>(qa + stage_base(st) + (long)s * TM * KS));
    unslice16(q, ya[st]);
  }
  auto values = [&](int st, double *x) {
    const double *g = gs + ((long)b * QBLK_STAGES + w * SPW + st) * KS + kc * 16;
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = (double)ya[st][i] * __ldg(g + i);
  };
  double mx = 0.0;
#pragma unroll
  for (int st = 0; st < SPW; ++st) {
    double x[16];
    values(st, x);
#pragma unroll
    for (int i = 0; i < 16; ++i) mx = fmax(mx, fabs(x[i]));
  }
  mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
  mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
  if (c < 8) smax[w][c] = mx;
  __syncthreads();
  mx = smax[0][r];
#pragma unroll
  for (int k = 1; k < kScaleWarps; ++k) mx = fmax(mx, smax[k][r]);
  const int sh = 30 - group_exponent(mx);
  if (w == 0 && c < 8) eb[(long)b * ebld + row] = ea[(long)row * nblk + b] + eg[b] - sh;
  const double scale = ldexp(1.0, sh);
#pragma unroll
  for (int st = 0; st < SPW; ++st) {
    double x[16];
    values(st, x);
    uint4 d[NSL];
    slice16(x, scale, d);
#pragma unroll
    for (int s = 0; s < NSL; ++s)
      *reinterpret_cast<uint4 *>(qb + stage_base(st) + (long)s * TM * KS) = d[s];
  }
}

__global__ void __launch_bounds__(32 * kScaleWarps)
scale_image_kernel(const int8_t *__restrict__ qa, int8_t *__restrict__ qb,
                   const double *__restrict__ gs, const int *__restrict__ ea,
                   const int *__restrict__ eg, int *__restrict__ eb, int nks, int nblk,
                   int ebld) {
  scale_image_body(qa, qb, gs, ea, eg, eb, nks, nblk, ebld, blockIdx.x, blockIdx.y);
}

// 2 K32 steps of one 64-wide stage: the kept digit products into their
// diagonal accumulators (column offset diagonal * N).  `fresh`: first stage
// of an accumulation, the first product of each diagonal overwrites.
template <int N, int NP, bool B5>
__device__ __forceinline__ void issue_stage(uint32_t tmem, uint32_t sa, uint32_t sb, bool fresh) {
  constexpr uint32_t idesc = idesc_i8(N);
#pragma unroll
  for (int kk = 0; kk < KS / 32; ++kk) {
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      const uint64_t ad = smem_desc(sa + prod_i(q, B5) * (TM * KS) + kk * 32 * 8);
      const uint64_t bd = smem_desc(sb + prod_j(q, B5) * (N * KS) + kk * 32 * 8);
      const bool first = fresh && kk == 0 && (q == 0 || prod_diag(q) != prod_diag(q - 1));
      umma_i8(tmem + (uint32_t)(prod_diag(q) * N), ad, bd, idesc, first ? 0u : 1u);
    }
  }
}

// ------------------------------------------------------------- quadrature
struct QuadArgs {
  const int8_t *a, *b;    // images of A and B, both in 128-row tiles
  const int *ea, *eb;     // exponents of A [row][nblk] and B [nblk][ebld]
  int nblk, nks;          // exponent blocks; stages per row tile (nblk * 64)
  int ebld;               // rows per block of eb
  int ntj;                // 96-column tiles
  int bpc;                // blocks per chunk
  int npair;
  double *work;           // [chunk][pair][128][96]
};

// Copies the 96 rows 96 J .. 96 J + 95 of stage ks of the B image (128-row
// tiles) into smem as a 96-row operand: per slice, the 12 row groups of 8
// rows lie in one or two tiles, each run contiguous.
__device__ __forceinline__ void copy_b96(uint8_t *dst, const int8_t *img, int J, long ks, int nks,
                                         uint64_t *bar) {
  const int g0 = 12 * J;                 // first row group
  const int t0 = g0 >> 4, r0 = g0 & 15;  // tile, group within the tile
  const int n0 = min(12, 16 - r0);       // groups in the first tile
#pragma unroll
  for (int s = 0; s < NSL; ++s) {
    uint8_t *d = dst + s * (QN * KS);
    const int8_t *src0 = img + ((long)t0 * nks + ks) * stage_bytes(TM) + s * (TM * KS) + r0 * 512;
    bulk_g2s(d, src0, n0 * 512, bar);
    if (n0 < 12) {
      const int8_t *src1 = img + ((long)(t0 + 1) * nks + ks) * stage_bytes(TM) + s * (TM * KS);
      bulk_g2s(d + n0 * 512, src1, (12 - n0) * 512, bar);
    }
  }
}

// CTA = (tile pair (I, J) with some nu >= mu, chunk of point blocks).
__device__ __forceinline__ void quad_i8_body(const QuadArgs &g, uint8_t *smem, int bx, int by) {
  __shared__ __align__(8) uint64_t full[NSTAGE], empty[NSTAGE], accfull, accempty, done;
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh, flag_sh;
  constexpr uint32_t A_BYTES = stage_bytes(TM), B_BYTES = stage_bytes(QN);
  constexpr uint32_t STAGE = A_BYTES + B_BYTES;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  volatile int *abort = &abort_sh;

  int I = 0, rem = bx;
  for (;;) {
    const int cnt = g.ntj - (4 * I) / 3;
    if (rem < cnt) break;
    rem -= cnt;
    ++I;
  }
  const int J = (4 * I) / 3 + rem;
  const int b0 = by * g.bpc;
  const int nb = max(0, min(b0 + g.bpc, g.nblk) - b0);

  if (t == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accfull, 1);
    mbar_init(&accempty, NEPI);
    mbar_init(&done, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kWarpM) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_sh)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_sh;

  if (warp == kWarpP) {
    if (lane == 0) {
      int it = 0;
      for (int bi = 0; bi < nb; ++bi) {
        bool ok = true;
        for (int st = 0; st < QBLK_STAGES; ++st) {
          const int slot = it % NSTAGE;
          if (!wait_phase(&empty[slot], ((it / NSTAGE) & 1) ^ 1, abort)) {
            ok = false;
            break;
          }
          const long ks = (long)(b0 + bi) * QBLK_STAGES + st;
          uint8_t *sa = smem + slot * STAGE;
          mbar_expect_tx(&full[slot], STAGE);
          bulk_g2s(sa, g.a + ((long)I * g.nks + ks) * A_BYTES, A_BYTES, &full[slot]);
          copy_b96(sa + A_BYTES, g.b, J, ks, g.nks, &full[slot]);
          ++it;
        }
        if (!ok) break;
      }
      // copies still in flight land before the CTA may exit
      for (int k = max(0, it - NSTAGE); k < it; ++k)
        wait_phase(&full[k % NSTAGE], (k / NSTAGE) & 1, nullptr);
    }
  } else if (warp == kWarpM) {
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int bi = 0; bi < nb && ok; ++bi) {
        if (!wait_phase(&accempty, (bi & 1) ^ 1, abort)) break;
        fence_after_sync();
        for (int st = 0; st < QBLK_STAGES; ++st, ++it) {
          const int slot = it % NSTAGE;
          if (!wait_phase(&full[slot], (it / NSTAGE) & 1, abort)) {
            ok = false;
            break;
          }
          fence_after_sync();
          const uint32_t sa = smem_u32(smem + slot * STAGE);
          issue_stage<QN, kQuadProducts, false>(tmem, sa, sa + A_BYTES, st == 0);
          umma_commit(&empty[slot]);
        }
        if (ok) umma_commit(&accfull);
      }
      umma_commit(&done);
    }
  } else {
    const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
    const int row = 32 * (warp & 3) + lane;
    const int col0 = DCW * (warp >> 2);
    const long mu = (long)I * TM + row;
    double part[DCW];
#pragma unroll
    for (int i = 0; i < DCW; ++i) part[i] = 0.0;
    bool ok = true;
    for (int bi = 0; bi < nb; ++bi) {
      if (!group_wait(&accfull, bi & 1, abort, &flag_sh, NEPI)) {
        ok = false;
        break;
      }
      fence_after_sync();
      const int blk = b0 + bi;
      const int ea = __ldg(g.ea + mu * g.nblk + blk);
      const int *eb = g.eb + (long)blk * g.ebld + J * QN + col0;  // DCW contiguous
#pragma unroll
      for (int c = 0; c < DCW; c += 8) {
        int32_t v[5][8];
#pragma unroll
        for (int d = 0; d < 5; ++d) tmem_ld8(tmem + lane_off + d * QN + col0 + c, v[d]);
        tmem_wait_ld();
#pragma unroll
        for (int d = 0; d < 5; ++d) tie8(v[d]);
        const int4 eb0 = __ldg(reinterpret_cast<const int4 *>(eb + c));
        const int4 eb1 = __ldg(reinterpret_cast<const int4 *>(eb + c + 4));
        const int ebv[8] = {eb0.x, eb0.y, eb0.z, eb0.w, eb1.x, eb1.y, eb1.z, eb1.w};
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const long long comb =
              (((((long long)v[0][i] * 256 + v[1][i]) * 256 + v[2][i]) * 256 + v[3][i]) * 256) +
              v[4][i];
          part[c + i] += (double)comb * pow2(ea + ebv[i] - 44);
        }
      }
      fence_before_sync();
      mbar_arrive(&accempty);
    }
    if (ok) {
      double *out = g.work + (((long)by * g.npair + bx) * TM + row) * QN + col0;
#pragma unroll
      for (int i = 0; i < DCW; ++i) out[i] = part[i];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == kWarpM) {
    if (lane == 0) wait_phase(&done, 0, nullptr);
    __syncwarp();
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
  }
}

__global__ void __launch_bounds__(NTHR, 1) quad_i8_kernel(QuadArgs g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  quad_i8_body(g, smem, blockIdx.x, blockIdx.y);
}

// F[mu][nu] = F[nu][mu] = sum over chunks (fixed order) of tile (mu/128, nu/96).
__device__ __forceinline__ void quad_i8_reduce_body(int n, int nchunk, int npair, int ntj,
                                                    const double *__restrict__ work,
                                                    double *__restrict__ F, int bx) {
  const long idx = (long)bx * blockDim.x + threadIdx.x;
  if (idx >= (long)n * n) return;
  const int mu = (int)(idx / n), nu = (int)(idx % n);
  if (mu > nu) return;
  const int I = mu / TM, J = nu / QN;
  int pair = 0;
  for (int i = 0; i < I; ++i) pair += ntj - (4 * i) / 3;
  pair += J - (4 * I) / 3;
  const double *w = work + ((long)pair * TM + mu % TM) * QN + nu % QN;
  const long stride = (long)npair * TM * QN;
  double s = 0.0;
  for (int c = 0; c < nchunk; ++c) s += w[c * stride];
  F[(long)mu * n + nu] = s;
  F[(long)nu * n + mu] = s;
}

__global__ void quad_i8_reduce_kernel(int n, int nchunk, int npair, int ntj,
                                      const double *__restrict__ work, double *__restrict__ F) {
  quad_i8_reduce_body(n, nchunk, npair, ntj, work, F, blockIdx.x);
}

// ---------------------------------------------------------------- density
// First 64-wide stage of nu that block m (functions 96 m .. 96 m + 95) of the
// density accumulates: the stage holding function 96 m.
__host__ __device__ constexpr int dens_first_stage(int m) { return m * DN / KS; }

// D' = the density matrix folded onto block-upper-triangular form, so that
// sum_{mu,nu} D'[mu][nu] phi_mu phi_nu = sum_{mu,nu} D[mu][nu] phi_mu phi_nu
// while block m needs only nu >= c(mu) = 64 dens_first_stage(mu / 96):
//   D'[mu][nu] = 0                        nu < c(mu)
//              = D[mu][nu] + D[nu][mu]    nu >= c(mu), mu < c(nu) (the mirror
//                                         entry is skipped by its block)
//              = D[mu][nu]                otherwise
// (for a symmetric D the sum is 2 D[mu][nu], exact).
__device__ __forceinline__ void dsym_body(const double *__restrict__ D, int n,
                                          double *__restrict__ out, int bx) {
  const long i = (long)bx * blockDim.x + threadIdx.x;
  if (i >= (long)n * n) return;
  const int mu = (int)(i / n), nu = (int)(i % n);
  const int cmu = dens_first_stage(mu / DN) * KS, cnu = dens_first_stage(nu / DN) * KS;
  double v = 0.0;
  if (nu >= cmu) {
    v = D[i];
    if (mu < cnu) v += D[(long)nu * n + mu];
  }
  out[i] = v;
}

__global__ void dsym_kernel(const double *__restrict__ D, int n, double *__restrict__ out) {
  dsym_body(D, n, out, blockIdx.x);
}

struct DensArgs {
  const int8_t *a;        // phi^T image [point tile][nks][slices][128 x 64]
  const int *ea;          // exponent per point
  const int8_t *d;        // D image [96-row tile][nks][5 slices][96 x 64]
  const int *ed;          // exponent per row of D
  int nks, nmt, npt, npoint;
  double *rho;
  const int *pidx;        // grid index of each (kept) point, or null
};

// Persistent: CTA c handles point tiles c, c + gridDim.x, ...  Pass (tile,
// m): T[p][mu] = sum_nu phi[nu][p] D'[mu][nu] for the 128 points and the 96
// functions of block m, accumulated in TMEM over nu >= 64 dens_first_stage(m)
// (D' is zero below, see dsym_kernel); the drain adds phi[mu][p] T[p][mu]
// into rho[p] (thread = point, DCW functions each).
__device__ __forceinline__ void density_i8_body(const DensArgs &g, uint8_t *smem, int bx,
                                                int gx) {
  __shared__ __align__(8) uint64_t full[NSTAGE], empty[NSTAGE], accfull, accempty, done;
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh, flag_sh;
  __shared__ double red[NEPI / 128][TM];
  constexpr uint32_t A_BYTES = stage_bytes(TM), B_BYTES = NSL_D * DN * KS;
  constexpr uint32_t STAGE = A_BYTES + B_BYTES;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  volatile int *abort = &abort_sh;

  if (t == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accfull, 1);
    mbar_init(&accempty, NEPI);
    mbar_init(&done, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kWarpM) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_sh)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_sh;

  if (warp == kWarpP) {
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int pt = bx; pt < g.npt && ok; pt += gx)
        for (int m = 0; m < g.nmt && ok; ++m)
          for (int ks = dens_first_stage(m); ks < g.nks; ++ks) {
            const int slot = it % NSTAGE;
            if (!wait_phase(&empty[slot], ((it / NSTAGE) & 1) ^ 1, abort)) {
              ok = false;
              break;
            }
            uint8_t *sa = smem + slot * STAGE;
            mbar_expect_tx(&full[slot], STAGE);
            bulk_g2s(sa, g.a + ((long)pt * g.nks + ks) * A_BYTES, A_BYTES, &full[slot]);
            bulk_g2s(sa + A_BYTES, g.d + ((long)m * g.nks + ks) * B_BYTES, B_BYTES, &full[slot]);
            ++it;
          }
      for (int k = max(0, it - NSTAGE); k < it; ++k)
        wait_phase(&full[k % NSTAGE], (k / NSTAGE) & 1, nullptr);
    }
  } else if (warp == kWarpM) {
    if (lane == 0) {
      int it = 0, pass = 0;
      bool ok = true;
      for (int pt = bx; pt < g.npt && ok; pt += gx)
        for (int m = 0; m < g.nmt && ok; ++m, ++pass) {
          if (!wait_phase(&accempty, (pass & 1) ^ 1, abort)) {
            ok = false;
            break;
          }
          fence_after_sync();
          const int ks0 = dens_first_stage(m);
          for (int ks = ks0; ks < g.nks; ++ks, ++it) {
            const int slot = it % NSTAGE;
            if (!wait_phase(&full[slot], (it / NSTAGE) & 1, abort)) {
              ok = false;
              break;
            }
            fence_after_sync();
            const uint32_t sa = smem_u32(smem + slot * STAGE);
            issue_stage<DN, kDensProducts, true>(tmem, sa, sa + A_BYTES, ks == ks0);
            umma_commit(&empty[slot]);
          }
          if (ok) umma_commit(&accfull);
        }
      umma_commit(&done);
    }
  } else {
    const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
    const int row = 32 * (warp & 3) + lane;
    const int h = warp >> 2;
    int pass = 0;
    bool ok = true;
    for (int pt = bx; pt < g.npt && ok; pt += gx) {
      const long p = (long)pt * TM + row;
      double acc = 0.0;
      for (int m = 0; m < g.nmt; ++m, ++pass) {
        if (!group_wait(&accfull, pass & 1, abort, &flag_sh, NEPI)) {
          ok = false;
          break;
        }
        fence_after_sync();
#pragma unroll 1
        for (int c = 0; c < DCW; c += 16) {
          int32_t v[5][16];
#pragma unroll
          for (int dg = 0; dg < 5; ++dg) {
            tmem_ld8(tmem + lane_off + dg * DN + DCW * h + c, v[dg]);
            tmem_ld8(tmem + lane_off + dg * DN + DCW * h + c + 8, v[dg] + 8);
          }
          tmem_wait_ld();
#pragma unroll
          for (int dg = 0; dg < 5; ++dg) {
            tie8(v[dg]);
            tie8(v[dg] + 8);
          }
          // functions mu0 .. mu0 + 15 lie in one 64-wide stage of phi^T
          const int mu0 = m * DN + DCW * h + c;
          if (mu0 < g.nks * KS) {
            const int8_t *pa = g.a + ((long)pt * g.nks + mu0 / KS) * A_BYTES +
                               core_off(row, mu0 % KS);
            uint4 q[NSL];
#pragma unroll
            for (int s = 0; s < NSL; ++s)
              q[s] = __ldg(reinterpret_cast<const uint4 *>(pa + (long)s * TM * KS));
            // exponents of D's rows mu0 .. mu0 + 15 (64-byte aligned)
            int edv[16];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const int4 t4 = __ldg(reinterpret_cast<const int4 *>(g.ed + mu0) + k);
              edv[4 * k] = t4.x;
              edv[4 * k + 1] = t4.y;
              edv[4 * k + 2] = t4.z;
              edv[4 * k + 3] = t4.w;
            }
            int yv[16];
            unslice16(q, yv);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int y = yv[i];
              const long long comb =
                  (((((long long)v[0][i] * 256 + v[1][i]) * 256 + v[2][i]) * 256 + v[3][i]) *
                   256) + v[4][i];
              acc = fma((double)y * pow2(edv[i]), (double)comb, acc);
            }
          }
        }
        fence_before_sync();
        mbar_arrive(&accempty);
      }
      if (!ok) break;
      red[h][row] = acc;
      named_sync(1, NEPI);
      if (h == 0 && p < g.npoint) {
        const int ep = __ldg(g.ea + p);
        double sum = red[0][row];
#pragma unroll
        for (int k = 1; k < NEPI / 128; ++k) sum += red[k][row];
        g.rho[g.pidx ? __ldg(g.pidx + p) : p] = sum * pow2(ep - 37) * pow2(ep - 37);
      }
      named_sync(1, NEPI);
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == kWarpM) {
    if (lane == 0) wait_phase(&done, 0, nullptr);
    __syncwarp();
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
  }
}

__global__ void __launch_bounds__(NTHR, 1) density_i8_kernel(DensArgs g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  density_i8_body(g, smem, blockIdx.x, gridDim.x);
}

int num_sms() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// rows_pad: rows written (a multiple of TR; rows >= nrows get zeros); ns
// slices (4 or 5).
cudaError_t launch_slice_rows(const double *src, long ld, int nrows, int rows_pad, int ncols,
                              const double *m1, const double *m2, int kb, int nblk, int TR,
                              int nks, int8_t *img, int *e, cudaStream_t s, int ns = NSL,
                              const int *cidx = nullptr) {
  if (ns == 5)
    slice_rows_kernel<5><<<dim3(rows_pad / 8, nblk), 256, 0, s>>>(
        src, ld, nrows, ncols, m1, m2, kb, nblk, TR, nks, img, e, cidx);
  else
    slice_rows_kernel<4><<<dim3(rows_pad / 8, nblk), 256, 0, s>>>(
        src, ld, nrows, ncols, m1, m2, kb, nblk, TR, nks, img, e, cidx);
  return cudaGetLastError();
}

// keep[p] = |wb w| max_mu phi[mu][p]^2 >= tol (1 for every point when
// tol <= 0); one thread per grid point, phi read once (coalesced over p).
__global__ void screen_kernel(const double *__restrict__ phi, long ld, int n, int npoint,
                              const double *__restrict__ wb, const double *__restrict__ w,
                              double tol, int *__restrict__ keep) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  if (!(tol > 0.0)) {
    keep[p] = 1;
    return;
  }
  double mx = 0.0;
  for (int mu = 0; mu < n; ++mu) mx = fmax(mx, fabs(__ldg(phi + (long)mu * ld + p)));
  const double t = fabs(wb[p] * w[p]);
  keep[p] = (t * mx) * mx >= tol ? 1 : 0;
}

}  // namespace

// ------------------------------------------------------------------- plan
struct Int8Plan {
  int n = 0, npoint = 0;  // npoint: kept points (all of the grid's without screening)
  int npoint_grid = 0;    // points of the grid
  long ld = 0;
  // quadrature: A and B images share 128-row tiles (nimg of them, enough for
  // the 96-row B tiles too)
  int nblk = 0, nks_q = 0, nti = 0, ntj = 0, nimg = 0, npair = 0, nchunk = 0, bpc = 0;
  // density
  int npt = 0, nks_d = 0, nmt = 0;
  int budget = 0;  // CTAs the kernels are sized for (the SM count by default)
  DevBuf<int8_t> qa, qb, da, dd;
  DevBuf<int> qa_e, qb_e, eg, da_e, dd_e;
  DevBuf<double> sc, isc, gs, work;
  DevBuf<double> dsym;  // D folded to block-upper-triangular form (density)
  DevBuf<int> keep;     // [npoint_grid] 1 for a kept point
  DevBuf<int> idx;      // [npoint] grid index of each kept point (screened plans)
  bool screened = false;
  unsigned long long serial = 0;  // unique per plan
};

// Sizes the kernels for `ctas` resident CTAs (<= 0: the SM count): the
// quadrature's chunks of point blocks minimise waves x blocks per chunk, the
// persistent density kernel runs min(point tiles, ctas) CTAs.  A smaller
// budget lets kernels of several plans share the GPU.
int int8_set_budget(Int8Plan *p, int ctas) {
  const int sms = ctas > 0 ? ctas : num_sms();
  long best = -1;
  int bpc_best = p->nblk, nchunk_best = 1;
  for (int nc = 1; nc <= p->nblk && nc <= 64; ++nc) {
    const int bpc = (p->nblk + nc - 1) / nc;
    const int used = (p->nblk + bpc - 1) / bpc;
    const long waves = ((long)p->npair * used + sms - 1) / sms;
    const long cost = waves * bpc;
    if (best < 0 || cost < best) {
      best = cost;
      bpc_best = bpc;
      nchunk_best = used;
    }
  }
  const size_t need = (size_t)nchunk_best * p->npair * TM * QN;
  if (need > p->work.n) NAPMO_TRY_CUDA(p->work.alloc(need), "alloc int8 workspace");
  p->bpc = bpc_best;
  p->nchunk = nchunk_best;
  p->budget = sms;
  return kOk;
}

int int8_plan_create(Int8Plan **out, int n, int npoint, const double *phi, long ld,
                     const double *wb, const double *w, double screen_tol, cudaStream_t s) {
  *out = nullptr;
  NAPMO_REQUIRE(n >= 1 && n <= 8192, "int8 contractions need 1 <= n <= 8192 basis functions");
  NAPMO_REQUIRE(npoint >= 1, "empty grid");
  static std::atomic<unsigned long long> next_serial{1};
  std::unique_ptr<Int8Plan> p(new Int8Plan);
  p->serial = next_serial++;
  p->n = n;
  p->npoint_grid = npoint;
  p->ld = ld;
  // point screening: keep flags, then the kept points' grid indices
  NAPMO_TRY_CUDA(p->keep.alloc(npoint), "alloc screening flags");
  screen_kernel<<<(npoint + 255) / 256, 256, 0, s>>>(phi, ld, n, npoint, wb, w, screen_tol,
                                                      p->keep.p);
  NAPMO_TRY_CUDA(cudaGetLastError(), "screen points");
  if (screen_tol > 0.0) {
    DevBuf<int> sel, cnt;
    DevBuf<uint8_t> tmp;
    NAPMO_TRY_CUDA(sel.alloc(npoint), "alloc screening");
    NAPMO_TRY_CUDA(cnt.alloc(1), "alloc screening");
    thrust::counting_iterator<int> first(0);
    size_t tb = 0;
    NAPMO_TRY_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, first, p->keep.p, sel.p, cnt.p,
                                              npoint, s),
                   "screening scan size");
    NAPMO_TRY_CUDA(tmp.alloc(tb + 1), "alloc screening");
    NAPMO_TRY_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, first, p->keep.p, sel.p, cnt.p,
                                              npoint, s),
                   "screening scan");
    int nkeep = 0;
    NAPMO_TRY_CUDA(cudaMemcpyAsync(&nkeep, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, s),
                   "screening count");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "screening");
    NAPMO_REQUIRE(nkeep >= 1, "point screening left no points");
    NAPMO_TRY_CUDA(p->idx.alloc(nkeep), "alloc kept points");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(p->idx.p, sel.p, nkeep * sizeof(int),
                                   cudaMemcpyDeviceToDevice, s),
                   "kept points");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "screening");
    npoint = nkeep;
    p->screened = true;
  }
  const int *pidx = p->screened ? p->idx.p : nullptr;
  p->npoint = npoint;
  p->nblk = (npoint + QKB - 1) / QKB;
  p->nks_q = p->nblk * QBLK_STAGES;
  p->nti = (n + TM - 1) / TM;
  p->ntj = (n + QN - 1) / QN;
  p->nimg = max(p->nti, (p->ntj * QN + TM - 1) / TM);
  p->npair = 0;
  for (int i = 0; i < p->nti; ++i) p->npair += p->ntj - (4 * i) / 3;
  p->npt = (int)(padded_points(npoint) / TM);
  const int npad64 = (n + KS - 1) / KS * KS;
  p->nks_d = npad64 / KS;
  p->nmt = (n + DN - 1) / DN;

  NAPMO_TRY_CUDA(p->sc.alloc(npoint), "alloc int8 scales");
  NAPMO_TRY_CUDA(p->isc.alloc(npoint), "alloc int8 scales");
  const size_t img_bytes = (size_t)p->nimg * p->nks_q * stage_bytes(TM);
  NAPMO_TRY_CUDA(p->qa.alloc(img_bytes), "alloc int8 phi image");
  NAPMO_TRY_CUDA(p->qa_e.alloc((size_t)p->nimg * TM * p->nblk), "alloc");
  NAPMO_TRY_CUDA(p->qb.alloc(img_bytes), "alloc int8 wv phi image");
  NAPMO_TRY_CUDA(cudaMemsetAsync(p->qb.p, 0, img_bytes, s), "zero int8 wv phi image");
  NAPMO_TRY_CUDA(p->qb_e.alloc((size_t)p->nimg * TM * p->nblk), "alloc");
  NAPMO_TRY_CUDA(cudaMemsetAsync(p->qb_e.p, 0, p->qb_e.n * sizeof(int), s), "zero");
  NAPMO_TRY_CUDA(p->eg.alloc(p->nblk), "alloc");
  NAPMO_TRY_CUDA(p->gs.alloc((size_t)p->nblk * QKB), "alloc");
  NAPMO_TRY_CUDA(p->da.alloc((size_t)p->npt * p->nks_d * stage_bytes(TM)), "alloc int8 phi^T image");
  NAPMO_TRY_CUDA(p->da_e.alloc((size_t)p->npt * TM), "alloc");
  NAPMO_TRY_CUDA(p->dd.alloc((size_t)p->nmt * p->nks_d * NSL_D * DN * KS), "alloc int8 D image");
  NAPMO_TRY_CUDA(p->dd_e.alloc((size_t)p->nmt * DN), "alloc");
  NAPMO_TRY_CUDA(p->dsym.alloc((size_t)n * n), "alloc folded D");

  int e = int8_set_budget(p.get(), 0);
  if (e) return e;
  balance_kernel<<<(npoint + 255) / 256, 256, 0, s>>>(npoint, wb, w, pidx, p->sc.p, p->isc.p);
  NAPMO_TRY_CUDA(cudaGetLastError(), "balance");
  NAPMO_TRY_CUDA(launch_slice_rows(phi, ld, n, p->nimg * TM, npoint, p->sc.p, nullptr, QKB,
                                   p->nblk, TM, p->nks_q, p->qa.p, p->qa_e.p, s, NSL, pidx),
                 "slice phi (quadrature)");
  slice_points_kernel<<<p->npt, TM, 0, s>>>(phi, ld, n, npoint, p->nks_d, p->da.p, p->da_e.p,
                                             pidx);
  NAPMO_TRY_CUDA(cudaGetLastError(), "slice phi (density)");
  *out = p.release();
  return kOk;
}

void int8_plan_destroy(Int8Plan *p) { delete p; }

size_t int8_plan_device_bytes(const Int8Plan *p) {
  return p->qa.n + p->qb.n + p->da.n + p->dd.n +
         4 * (p->qa_e.n + p->qb_e.n + p->eg.n + p->da_e.n + p->dd_e.n) +
         4 * (p->keep.n + p->idx.n) +
         8 * (p->sc.n + p->isc.n + p->gs.n + p->work.n + p->dsym.n);
}

int int8_plan_npoint(const Int8Plan *p) { return p->npoint; }

const int *int8_plan_keep(const Int8Plan *p) { return p->screened ? p->keep.p : nullptr; }

unsigned long long int8_plan_serial(const Int8Plan *p) { return p->serial; }

int int8_density(Int8Plan *p, const double *D, double *rho, cudaStream_t s) {
  const long nn = (long)p->n * p->n;
  dsym_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(D, p->n, p->dsym.p);
  NAPMO_TRY_CUDA(cudaGetLastError(), "fold D");
  NAPMO_TRY_CUDA(launch_slice_rows(p->dsym.p, p->n, p->n, p->nmt * DN, p->n, nullptr, nullptr,
                                   p->nks_d * KS, 1, DN, p->nks_d, p->dd.p, p->dd_e.p, s, NSL_D),
                 "slice D");
  if (p->screened)  // dropped points get rho = 0
    NAPMO_TRY_CUDA(cudaMemsetAsync(rho, 0, (size_t)p->npoint_grid * sizeof(double), s), "rho");
  DensArgs g{p->da.p, p->da_e.p, p->dd.p, p->dd_e.p, p->nks_d, p->nmt, p->npt, p->npoint, rho,
             p->screened ? p->idx.p : nullptr};
  const int smem = NSTAGE * (stage_bytes(TM) + NSL_D * DN * KS);
  NAPMO_TRY_CUDA(cudaFuncSetAttribute(density_i8_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                 "density_i8 smem");
  const int grid = p->npt < p->budget ? p->npt : p->budget;
  density_i8_kernel<<<grid, NTHR, smem, s>>>(g);
  NAPMO_TRY_CUDA(cudaGetLastError(), "density_i8");
  return kOk;
}

int int8_quadrature(Int8Plan *p, const double *phi, const double *wv, double *F,
                    cudaStream_t s) {
  (void)phi;
  gscale_kernel<<<p->nblk, 256, 0, s>>>(p->npoint, wv, p->isc.p,
                                        p->screened ? p->idx.p : nullptr, p->gs.p, p->eg.p);
  NAPMO_TRY_CUDA(cudaGetLastError(), "block scales");
  scale_image_kernel<<<dim3((p->n + 7) / 8, p->nblk), 32 * kScaleWarps, 0, s>>>(
      p->qa.p, p->qb.p, p->gs.p, p->qa_e.p, p->eg.p, p->qb_e.p, p->nks_q, p->nblk,
      p->nimg * TM);
  NAPMO_TRY_CUDA(cudaGetLastError(), "wv phi image");
  QuadArgs g{p->qa.p, p->qb.p, p->qa_e.p, p->qb_e.p, p->nblk, p->nks_q, p->nimg * TM,
             p->ntj,  p->bpc,  p->npair, p->work.p};
  const int smem = NSTAGE * (stage_bytes(TM) + stage_bytes(QN));
  NAPMO_TRY_CUDA(cudaFuncSetAttribute(quad_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem),
                 "quad_i8 smem");
  quad_i8_kernel<<<dim3(p->npair, p->nchunk), NTHR, smem, s>>>(g);
  NAPMO_TRY_CUDA(cudaGetLastError(), "quad_i8");
  const long nn = (long)p->n * p->n;
  quad_i8_reduce_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(p->n, p->nchunk, p->npair,
                                                                     p->ntj, p->work.p, F);
  NAPMO_TRY_CUDA(cudaGetLastError(), "quad_i8 reduce");
  return kOk;
}

// ------------------------------------------------------------- stage batches
// The int8 build stages of many plans as one launch each: a batched launch
// runs the sum of the molecules' own grids; CTA b belongs to the molecule m
// with cta_off[m] <= b < cta_off[m + 1] and runs the kernel's body with its
// local block index (x = local % gx[m], y = local / gx[m]), so every
// molecule's arithmetic and launch shape are those of its own plan.  The
// persistent density keeps each molecule's own CTA count as its tile stride.
namespace {

struct BatchMap {
  const int *cta_off;  // [nmol + 1]
  const int *gx;       // [nmol] x extent of the molecule's own grid
  int nmol;
};

__device__ __forceinline__ int map_cta(const BatchMap &m, int *bx, int *by) {
  const int b = blockIdx.x;
  int lo = 0, hi = m.nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (m.cta_off[mid] <= b) lo = mid; else hi = mid - 1;
  }
  const int local = b - m.cta_off[lo], gx = m.gx[lo];
  *bx = local % gx;
  *by = local / gx;
  return lo;
}

struct DsymArg { const double *D; double *out; int n; };
struct SliceArg {
  const double *src; long ld; int nrows, ncols, kb, nblk, TR, nks;
  int8_t *img; int *e;
};
struct GscaleArg { const double *wv, *isc; const int *pidx; double *gs; int *eg; int npoint; };
struct ScaleArg {
  const int8_t *qa; int8_t *qb; const double *gs; const int *ea, *eg; int *eb;
  int nks, nblk, ebld;
};
struct ReduceArg { const double *work; double *F; int n, nchunk, npair, ntj; };

__global__ void dsym_batch_kernel(const DsymArg *__restrict__ a, BatchMap m) {
  int bx, by;
  const DsymArg g = a[map_cta(m, &bx, &by)];
  dsym_body(g.D, g.n, g.out, bx);
}

__global__ void __launch_bounds__(256) slice_d_batch_kernel(const SliceArg *__restrict__ a,
                                                            BatchMap m) {
  int bx, by;
  const SliceArg g = a[map_cta(m, &bx, &by)];
  slice_rows_body<NSL_D>(g.src, g.ld, g.nrows, g.ncols, nullptr, nullptr, g.kb, g.nblk, g.TR,
                         g.nks, g.img, g.e, nullptr, bx, by);
}

__global__ void __launch_bounds__(NTHR, 1) density_i8_batch_kernel(const DensArgs *__restrict__ a,
                                                                   BatchMap m) {
  extern __shared__ __align__(1024) uint8_t smem[];
  int bx, by;
  const int mol = map_cta(m, &bx, &by);
  density_i8_body(a[mol], smem, bx, m.gx[mol]);
}

__global__ void __launch_bounds__(256) gscale_batch_kernel(const GscaleArg *__restrict__ a,
                                                           BatchMap m) {
  int bx, by;
  const GscaleArg g = a[map_cta(m, &bx, &by)];
  gscale_body(g.npoint, g.wv, g.isc, g.pidx, g.gs, g.eg, bx);
}

__global__ void __launch_bounds__(32 * kScaleWarps) scale_image_batch_kernel(const ScaleArg *__restrict__ a,
                                                                BatchMap m) {
  int bx, by;
  const ScaleArg g = a[map_cta(m, &bx, &by)];
  scale_image_body(g.qa, g.qb, g.gs, g.ea, g.eg, g.eb, g.nks, g.nblk, g.ebld, bx, by);
}

__global__ void __launch_bounds__(NTHR, 1) quad_i8_batch_kernel(const QuadArgs *__restrict__ a,
                                                                BatchMap m) {
  extern __shared__ __align__(1024) uint8_t smem[];
  int bx, by;
  const int mol = map_cta(m, &bx, &by);
  quad_i8_body(a[mol], smem, bx, by);
}

__global__ void quad_i8_reduce_batch_kernel(const ReduceArg *__restrict__ a, BatchMap m) {
  int bx, by;
  const ReduceArg g = a[map_cta(m, &bx, &by)];
  quad_i8_reduce_body(g.n, g.nchunk, g.npair, g.ntj, g.work, g.F, bx);
}

// Per-molecule grids (gx x gy) of one batched launch: prefix CTA offsets and
// x extents on the device, total CTAs in *total.
struct LaunchMap {
  DevBuf<int> off, gx;
  int total = 0, nmol = 0;
  int build(const std::vector<int> &gxs, const std::vector<int> &gys, cudaStream_t s) {
    std::vector<int> o(1, 0);
    for (size_t i = 0; i < gxs.size(); ++i) o.push_back(o.back() + gxs[i] * gys[i]);
    total = o.back();
    nmol = (int)gxs.size();
    NAPMO_TRY_CUDA(off.upload(o, s), "batch map");
    NAPMO_TRY_CUDA(gx.upload(gxs, s), "batch map");
    return kOk;
  }
  BatchMap map() const { return BatchMap{off.p, gx.p, nmol}; }
};

}  // namespace

struct Int8Batch {
  int nmol = 0;
  DevBuf<DsymArg> dsym;
  DevBuf<SliceArg> slice;
  DevBuf<DensArgs> dens;
  DevBuf<GscaleArg> gscale;
  DevBuf<ScaleArg> scale;
  DevBuf<QuadArgs> quad;
  DevBuf<ReduceArg> reduce;
  LaunchMap m_dsym, m_slice, m_dens, m_gscale, m_scale, m_quad, m_reduce;
};

// Tables of the batched int8 stages: molecule m reads D[m], writes rho[m]
// (its kept points scattered by the plan's index; the caller zeroes rho
// first), reads wv[m] (zero padded) and writes F[m].
int int8_batch_new(const std::vector<Int8Plan *> &plans, const std::vector<const double *> &D,
                   const std::vector<double *> &rho, const std::vector<const double *> &wv,
                   const std::vector<double *> &F, cudaStream_t s, Int8Batch **out) {
  std::unique_ptr<Int8Batch> b(new Int8Batch);
  const int nmol = (int)plans.size();
  b->nmol = nmol;
  std::vector<DsymArg> ds(nmol);
  std::vector<SliceArg> sl(nmol);
  std::vector<DensArgs> de(nmol);
  std::vector<GscaleArg> gs(nmol);
  std::vector<ScaleArg> sc(nmol);
  std::vector<QuadArgs> qa(nmol);
  std::vector<ReduceArg> re(nmol);
  std::vector<int> gx[7], gy[7];
  for (int m = 0; m < nmol; ++m) {
    Int8Plan *p = plans[m];
    const long nn = (long)p->n * p->n;
    ds[m] = DsymArg{D[m], p->dsym.p, p->n};
    gx[0].push_back((int)((nn + 255) / 256));
    gy[0].push_back(1);
    sl[m] = SliceArg{p->dsym.p, p->n, p->n, p->n, p->nks_d * KS, 1, DN, p->nks_d, p->dd.p,
                     p->dd_e.p};
    gx[1].push_back(p->nmt * DN / 8);
    gy[1].push_back(1);
    de[m] = DensArgs{p->da.p, p->da_e.p, p->dd.p, p->dd_e.p, p->nks_d, p->nmt, p->npt,
                     p->npoint, rho[m], p->screened ? p->idx.p : nullptr};
    gx[2].push_back(std::max(1, std::min(p->npt, p->budget)));
    gy[2].push_back(p->npt > 0 ? 1 : 0);
    gs[m] = GscaleArg{wv[m], p->isc.p, p->screened ? p->idx.p : nullptr, p->gs.p, p->eg.p,
                      p->npoint};
    gx[3].push_back(p->nblk);
    gy[3].push_back(1);
    sc[m] = ScaleArg{p->qa.p, p->qb.p, p->gs.p, p->qa_e.p, p->eg.p, p->qb_e.p, p->nks_q,
                     p->nblk, p->nimg * TM};
    gx[4].push_back((p->n + 7) / 8);
    gy[4].push_back(p->nblk);
    qa[m] = QuadArgs{p->qa.p, p->qb.p, p->qa_e.p, p->qb_e.p, p->nblk, p->nks_q, p->nimg * TM,
                     p->ntj, p->bpc, p->npair, p->work.p};
    gx[5].push_back(p->npair);
    gy[5].push_back(p->nchunk);
    re[m] = ReduceArg{p->work.p, F[m], p->n, p->nchunk, p->npair, p->ntj};
    gx[6].push_back((int)((nn + 255) / 256));
    gy[6].push_back(1);
  }
  NAPMO_TRY_CUDA(b->dsym.upload(ds, s), "batch tables");
  NAPMO_TRY_CUDA(b->slice.upload(sl, s), "batch tables");
  NAPMO_TRY_CUDA(b->dens.upload(de, s), "batch tables");
  NAPMO_TRY_CUDA(b->gscale.upload(gs, s), "batch tables");
  NAPMO_TRY_CUDA(b->scale.upload(sc, s), "batch tables");
  NAPMO_TRY_CUDA(b->quad.upload(qa, s), "batch tables");
  NAPMO_TRY_CUDA(b->reduce.upload(re, s), "batch tables");
  LaunchMap *maps[7] = {&b->m_dsym, &b->m_slice, &b->m_dens, &b->m_gscale, &b->m_scale,
                        &b->m_quad, &b->m_reduce};
  for (int k = 0; k < 7; ++k) {
    const int e = maps[k]->build(gx[k], gy[k], s);
    if (e) return e;
  }
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch tables");
  *out = b.release();
  return kOk;
}

void int8_batch_free(Int8Batch *b) { delete b; }

// D -> D' (folded) -> 5-digit image -> rho of every molecule (rho zeroed by
// the caller).
int int8_batch_density(Int8Batch *b, cudaStream_t s) {
  if (b->m_dsym.total)
    dsym_batch_kernel<<<b->m_dsym.total, 256, 0, s>>>(b->dsym.p, b->m_dsym.map());
  NAPMO_TRY_CUDA(cudaGetLastError(), "fold D");
  if (b->m_slice.total)
    slice_d_batch_kernel<<<b->m_slice.total, 256, 0, s>>>(b->slice.p, b->m_slice.map());
  NAPMO_TRY_CUDA(cudaGetLastError(), "slice D");
  const int smem = NSTAGE * (stage_bytes(TM) + NSL_D * DN * KS);
  NAPMO_TRY_CUDA(cudaFuncSetAttribute(density_i8_batch_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                 "density_i8 smem");
  if (b->m_dens.total)
    density_i8_batch_kernel<<<b->m_dens.total, NTHR, smem, s>>>(b->dens.p, b->m_dens.map());
  NAPMO_TRY_CUDA(cudaGetLastError(), "density_i8");
  return kOk;
}

// wv -> block scales -> B images -> F of every molecule.
int int8_batch_quadrature(Int8Batch *b, cudaStream_t s) {
  if (b->m_gscale.total)
    gscale_batch_kernel<<<b->m_gscale.total, 256, 0, s>>>(b->gscale.p, b->m_gscale.map());
  NAPMO_TRY_CUDA(cudaGetLastError(), "block scales");
  if (b->m_scale.total)
    scale_image_batch_kernel<<<b->m_scale.total, 32 * kScaleWarps, 0, s>>>(b->scale.p,
                                                                          b->m_scale.map());
  NAPMO_TRY_CUDA(cudaGetLastError(), "wv phi image");
  const int smem = NSTAGE * (stage_bytes(TM) + stage_bytes(QN));
  NAPMO_TRY_CUDA(cudaFuncSetAttribute(quad_i8_batch_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                 "quad_i8 smem");
  if (b->m_quad.total)
    quad_i8_batch_kernel<<<b->m_quad.total, NTHR, smem, s>>>(b->quad.p, b->m_quad.map());
  NAPMO_TRY_CUDA(cudaGetLastError(), "quad_i8");
  if (b->m_reduce.total)
    quad_i8_reduce_batch_kernel<<<b->m_reduce.total, 256, 0, s>>>(b->reduce.p,
                                                                  b->m_reduce.map());
  NAPMO_TRY_CUDA(cudaGetLastError(), "quad_i8 reduce");
  return kOk;
}

// Exercises the bounded waits of the tensor-core kernels without a fault: one
// role (thread 0) waits on an mbarrier that nothing arrives on, with the
// kernels' own wait_phase (limit kTimeoutNs, then kDeviceTimeout in
// g_tc_error and the abort flag set); a second role (thread 32) waits on
// another such barrier and must leave through the abort flag, as the roles of
// density_i8 / quad_i8 do.  out[0], out[1]: the two waits' results (0 = gave
// up).
namespace {
__global__ void tc_wait_selftest_kernel(int *out) {
  __shared__ __align__(8) uint64_t never[2];
  __shared__ int abort_sh;
  volatile int *abort = &abort_sh;
  if (threadIdx.x == 0) {
    mbar_init(&never[0], 1);
    mbar_init(&never[1], 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) out[0] = wait_phase(&never[0], 0, abort) ? 1 : 0;
  if (threadIdx.x == 32) out[1] = wait_phase(&never[1], 0, abort) ? 1 : 0;
  __syncthreads();
}
}  // namespace

int tc_wait_selftest(int *out_dev, cudaStream_t s) {
  tc_wait_selftest_kernel<<<1, 64, 0, s>>>(out_dev);
  NAPMO_TRY_CUDA(cudaGetLastError(), "wait self-test");
  return kOk;
}

int tc_error_status(cudaStream_t s, bool reset) {
  int h = 0;
  if (cudaMemcpyFromSymbolAsync(&h, g_tc_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s) !=
      cudaSuccess)
    return kCudaError;
  cudaStreamSynchronize(s);
  if (reset && h) {
    const int z = 0;
    cudaMemcpyToSymbolAsync(g_tc_error, &z, sizeof(int), 0, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
  }
  return h;
}

}  // namespace napmo
