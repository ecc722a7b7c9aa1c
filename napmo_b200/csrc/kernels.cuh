// Kernel launchers of the napmo_b200 CUDA library (sm_100a).
#pragma once
#include <vector>

#include <cuda_runtime.h>

#include "device_types.h"

namespace napmo {

// Becke partition weights (becke.cu).  R_ij and a_ij are the packed
// lower-triangular inter-atomic distances and size adjustments of nAPMO
// (src/grid/becke.cpp:80-115), computed on the host.
cudaError_t launch_becke_weights(int npoint, int ncenter, const double *x,
                                 const double *y, const double *z,
                                 const double *origin, const double *Rij,
                                 const double *aij, const int *atom_offset,
                                 double *out, cudaStream_t s);

// Contracted Cartesian GTO values phi[f * ld + p] (gto.cu); with `grad`
// non-null also d/dx, d/dy, d/dz as three further [nfunc][ld] planes.
cudaError_t launch_basis_values(const DeviceBasis &b, int npoint, const double *x,
                                const double *y, const double *z, double *phi,
                                long ld, double *grad, cudaStream_t s);

// FP64 quadratures (quad.cu).
//   rho[p] = sum_{mu,nu} D[mu][nu] phi[mu][p] phi[nu][p]
//   F[mu][nu] = sum_p phi[mu][p] wv[p] phi[nu][p]  (upper triangle mirrored)
size_t density_workspace_bytes(int n, int npoint);
// groups / ngroup (optional): only these 128-point groups are computed (the
// rest of rho is zeroed); keep (optional): rho = 0 at dropped points.
cudaError_t launch_density_f64(int n, int npoint, const double *phi, long ld,
                               const double *D, double *rho, cudaStream_t s,
                               const int *groups = nullptr, int ngroup = 0,
                               const int *keep = nullptr);
size_t quadrature_workspace_bytes(int n, int npoint);
// `phib` (default phi) is the second operand; wv must be zero-padded to the
// next multiple of 128 points and phi rows zero beyond npoint.  blocks /
// nblock (optional): the sum runs over these 16-point blocks only.
cudaError_t launch_quadrature_f64(int n, int npoint, const double *phi, long ld,
                                  const double *wv, double *F, double *work,
                                  cudaStream_t s, const double *phib = nullptr,
                                  const int *blocks = nullptr, int nblock = 0);
// Batched FP64 launches (one launch per stage for many molecules).
struct DensBatchArg {      // density of one molecule
  const double *phi;       // [n][ld]
  long ld;
  const double *D;         // [n][n]
  double *rho;             // [npoint]
  const int *keep;         // screening flags or null
  int n, npoint, vecD, pad;
};
struct QuadBatchArg {      // quadrature of one molecule
  const double *phi;       // [n][ld]
  long ld;
  const double *wv;        // zero padded to npoint rounded up to 128
  double *work;            // [nchunk][tile][128][128]
  double *F;               // [n][n]
  const int *blocks;       // 16-point blocks of a screened plan, or null
  int n, npad, nblk, chunk, nchunk;
};
struct WeightBatchArg {    // wv = wb w (q v), zero padded to npad
  const double *wb, *w, *v;
  double *wv;
  int npoint, npad;
};
// Device work queue of a persistent batched launch: items[i] = (molecule,
// tile, chunk, -); item i is taken once *posted > i, waiting at most
// timeout_ns; a timeout records kDeviceTimeout in *status.
struct BatchQueue {
  const int4 *items;
  int nitems;
  int *head;
  const int *posted;
  int *status;
  unsigned long long timeout_ns;
};
// Split-K chunking of a K range of npad points in a workspace sized for a grid
// of pad_full points (quadrature_workspace_bytes): chunk count <= the grid's.
int quadrature_chunking(int n, int npad, int *chunk, int pad_full);
cudaError_t launch_density_batch(const DensBatchArg *args, const BatchQueue &q, int grid,
                                 cudaStream_t s);
cudaError_t launch_quadrature_batch(const QuadBatchArg *args, const BatchQueue &q, int grid,
                                    cudaStream_t s);
cudaError_t launch_quadrature_reduce_batch(const QuadBatchArg *args, int nmol, cudaStream_t s);
cudaError_t launch_combine_weights_batch(const WeightBatchArg *args, int nmol, double q,
                                         cudaStream_t s);
// FP64 point screening: keep[p] (|wb w| max_mu phi_mu(p)^2 >= tol), and the
// flags of the 16-point blocks and 128-point groups holding a kept point.
cudaError_t launch_fp64_screening(int n, int npoint, const double *phi, long ld, const double *wb,
                                  const double *w, double tol, int *keep, int *block_flags,
                                  int *group_flags, cudaStream_t s);
inline long padded_points(int npoint) { return ((long)npoint + 127) / 128 * 128; }
// Combined quadrature weight wv[p] = wb[p] * w[p] * (q * v[p] + vext[p]).
cudaError_t launch_combine_weights(int npoint, const double *wb, const double *w,
                                   double q, const double *v, const double *vext,
                                   double *wv, cudaStream_t s);

// Adds nchunk partial 128x128 upper-triangle tiles [chunk][tile][128][128]
// in fixed order and writes both triangles of F.
cudaError_t launch_quadrature_reduce(int n, int nchunk, const double *work, double *F,
                                     cudaStream_t s);

// Int8-slice tensor-core quadratures (tc.cu).  A plan holds phi's operand
// images (built once from phi, wb and w) and the per-call scratch; the calls
// return library status codes and record g_tc_error on a device timeout.
struct Int8Plan;
// screen_tol > 0 keeps only the points with |wb w| max_mu phi_mu^2 >= screen_tol
// (rho is 0 at the others, which the quadrature skips).
int int8_plan_create(Int8Plan **out, int n, int npoint, const double *phi, long ld,
                     const double *wb, const double *w, double screen_tol, cudaStream_t s);
void int8_plan_destroy(Int8Plan *p);
// Points the plan keeps, and their flags over the grid (null without screening).
int int8_plan_npoint(const Int8Plan *p);
const int *int8_plan_keep(const Int8Plan *p);
// Unique, never reused number of the plan (names its screening mask).
unsigned long long int8_plan_serial(const Int8Plan *p);
// CTA budget the int8 kernels are sized for (<= 0: the SM count).
int int8_set_budget(Int8Plan *p, int ctas);
size_t int8_plan_device_bytes(const Int8Plan *p);
int int8_density(Int8Plan *p, const double *D, double *rho, cudaStream_t s);
int int8_quadrature(Int8Plan *p, const double *phi, const double *wv, double *F,
                    cudaStream_t s);
// Returns the device error word of the tensor-core kernels (0 = none), after
// synchronising `s`; `reset` clears it.
int tc_error_status(cudaStream_t s, bool reset);
int tc_wait_selftest(int *out_dev, cudaStream_t s);
// int8 build stages of many plans, one batched launch each (see tc.cu).
struct Int8Batch;
int int8_batch_new(const std::vector<Int8Plan *> &plans, const std::vector<const double *> &D,
                   const std::vector<double *> &rho, const std::vector<const double *> &wv,
                   const std::vector<double *> &F, cudaStream_t s, Int8Batch **out);
void int8_batch_free(Int8Batch *b);
int int8_batch_density(Int8Batch *b, cudaStream_t s);
int int8_batch_quadrature(Int8Batch *b, cudaStream_t s);

}  // namespace napmo
