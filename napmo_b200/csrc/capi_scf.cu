// The FP64 SCF step next to the Fock build (nAPMO src/wavefunction/
// wavefunction.cpp:12-166): generalised eigenproblem F C = S C e by cuSOLVER
// (dsygvd, FP64, on the device), density D = eta C_occ C_occ^T, energy
// sum D o (H + G/2 + J) + E_xc and rmsd ||D - D_old||_F by device kernels.
// Also the common-point index between species grids (src/grid/
// multi_grid.cpp:37-86) and error-raising stubs for the libint-based
// analytic integrals and the auxiliary Slater basis, which are not part of
// the grid-quadrature path.
#include <cusolverDn.h>

#include <map>
#include <vector>

#include "capi_common.cuh"
#include "host.h"
#include "wavefunction.h"

namespace napmo {

namespace {

// C_rowmajor[i][k] = A_colmajor[k][i]
__global__ void colmajor_to_rowmajor(int n, const double *A, double *C) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  const int i = e / n, k = e % n;
  C[e] = A[(long)k * n + i];
}

// D[i][j] = eta sum_{k < occ} C[i][k] C[j][k]
__global__ void density_from_c(int n, int occ, double eta, const double *C, double *D) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  const int i = e / n, j = e % n;
  double s = 0.0;
  for (int k = 0; k < occ; ++k) s += C[(long)i * n + k] * C[(long)j * n + k];
  D[e] = s * eta;
}

// out[0] = sum D (H + 0.5 G + J), out[1] = sum (D - L)^2  (fixed order)
__global__ void energy_rmsd(int n, const double *D, const double *H, const double *G,
                            const double *J, const double *L, double *out) {
  __shared__ double se[256], sr[256];
  double e = 0.0, r = 0.0;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
    e += D[i] * (H[i] + 0.5 * G[i] + J[i]);
    if (L) {
      const double d = D[i] - L[i];
      r += d * d;
    }
  }
  se[threadIdx.x] = e;
  sr[threadIdx.x] = r;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      se[threadIdx.x] += se[threadIdx.x + o];
      sr[threadIdx.x] += sr[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = se[0];
    out[1] = sr[0];
  }
}

cusolverDnHandle_t solver_handle() {
  static thread_local std::map<int, cusolverDnHandle_t> handles;
  int dev = 0;
  cudaGetDevice(&dev);
  auto it = handles.find(dev);
  if (it != handles.end()) return it->second;
  cusolverDnHandle_t h = nullptr;
  if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return nullptr;
  handles[dev] = h;
  return h;
}

}  // namespace

// Solves F C = S C e (device, row-major symmetric inputs); C row-major with
// eigenvectors in columns, e ascending.  Fd and Sd are overwritten.
int gen_eigh_device(int n, double *Fd, double *Sd, double *Cd, double *Ed, cudaStream_t s) {
  cusolverDnHandle_t h = solver_handle();
  if (!h) return set_error(kCudaError, "cusolverDnCreate failed");
  cusolverDnSetStream(h, s);
  int lwork = 0;
  if (cusolverDnDsygvd_bufferSize(h, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                  CUBLAS_FILL_MODE_LOWER, n, Fd, n, Sd, n, Ed, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    return set_error(kCudaError, "dsygvd buffer size failed");
  DevBuf<double> work;
  DevBuf<int> info;
  NAPMO_TRY_CUDA(work.alloc(lwork > 0 ? lwork : 1), "eigh workspace");
  NAPMO_TRY_CUDA(info.alloc(1), "eigh info");
  if (cusolverDnDsygvd(h, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                       n, Fd, n, Sd, n, Ed, work.p, lwork, info.p) != CUSOLVER_STATUS_SUCCESS)
    return set_error(kCudaError, "dsygvd failed");
  int hinfo = 0;
  NAPMO_TRY_CUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "eigh");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "eigh");
  if (hinfo != 0) return set_error(kInvalidArgument, "dsygvd: info = " + std::to_string(hinfo));
  colmajor_to_rowmajor<<<(n * n + 255) / 256, 256, 0, s>>>(n, Fd, Cd);
  NAPMO_TRY_CUDA(cudaGetLastError(), "eigh");
  return kOk;
}

// Diagonalise (A, S) for a WaveFunction and form C, O and (optionally) D.
static int diag_and_density(WaveFunction *psi, const double *A, bool form_density,
                            double energy_out[2], bool with_energy) {
  cudaStream_t s = host_api_stream();
  const int n = psi->ndim;
  const size_t nn = (size_t)n * n;
  DevBuf<double> F, S, C, E, D, H, G, J, L, out;
  NAPMO_TRY_CUDA(F.upload(A, nn, s), "upload");
  NAPMO_TRY_CUDA(S.upload(psi->S, nn, s), "upload");
  NAPMO_TRY_CUDA(C.alloc(nn), "alloc");
  NAPMO_TRY_CUDA(E.alloc(n), "alloc");
  int st = gen_eigh_device(n, F.p, S.p, C.p, E.p, s);
  if (st) return st;
  NAPMO_TRY_CUDA(cudaMemcpyAsync(psi->C, C.p, nn * sizeof(double), cudaMemcpyDeviceToHost, s), "C");
  NAPMO_TRY_CUDA(cudaMemcpyAsync(psi->O, E.p, n * sizeof(double), cudaMemcpyDeviceToHost, s), "O");
  if (form_density) {
    NAPMO_TRY_CUDA(D.alloc(nn), "alloc");
    density_from_c<<<(int)((nn + 255) / 256), 256, 0, s>>>(n, psi->occupation, psi->eta, C.p, D.p);
    NAPMO_TRY_CUDA(cudaMemcpyAsync(psi->D, D.p, nn * sizeof(double), cudaMemcpyDeviceToHost, s),
                   "D");
    if (with_energy) {
      NAPMO_TRY_CUDA(H.upload(psi->H, nn, s), "upload");
      NAPMO_TRY_CUDA(G.upload(psi->G, nn, s), "upload");
      NAPMO_TRY_CUDA(J.upload(psi->J, nn, s), "upload");
      NAPMO_TRY_CUDA(L.upload(psi->L, nn, s), "upload");
      NAPMO_TRY_CUDA(out.alloc(2), "alloc");
      energy_rmsd<<<1, 256, 0, s>>>(n, D.p, H.p, G.p, J.p, L.p, out.p);
      NAPMO_TRY_CUDA(cudaMemcpyAsync(energy_out, out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                     s),
                     "energy");
    }
  }
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "sync");
  return kOk;
}

// --------------------------------------------------------- common points
struct MultiGrid {
  int nspecies = 0;
  std::vector<BeckeGrid *> grids;
  std::map<std::pair<int, int>, std::vector<int>> index;
};

__global__ void common_count(long na, long nb, const double *A, const double *B, int *cnt) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= na) return;
  const double x = A[3 * i], y = A[3 * i + 1], z = A[3 * i + 2];
  int c = 0;
  for (long j = 0; j < nb; ++j)
    if (x == B[3 * j] && y == B[3 * j + 1] && z == B[3 * j + 2]) ++c;
  cnt[i] = c;
}

__global__ void common_write(long na, long nb, const double *A, const double *B,
                             const long *start, int *pairs) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= na) return;
  const double x = A[3 * i], y = A[3 * i + 1], z = A[3 * i + 2];
  long o = start[i];
  for (long j = 0; j < nb; ++j)
    if (x == B[3 * j] && y == B[3 * j + 1] && z == B[3 * j + 2]) {
      pairs[2 * o] = (int)i;
      pairs[2 * o + 1] = (int)j;
      ++o;
    }
}

// Pairs (i in the larger grid, j in the smaller) of bit-identical points, in
// the reference's order (i ascending, then j ascending).
static int common_points(const BeckeGrid *a, const BeckeGrid *b, std::vector<int> &out) {
  if (b->size > a->size) std::swap(a, b);
  cudaStream_t s = host_api_stream();
  const long na = a->size, nb = b->size;
  DevBuf<double> dA, dB;
  DevBuf<int> cnt, pairs;
  DevBuf<long> start;
  NAPMO_TRY_CUDA(dA.upload(a->points, s), "common");
  NAPMO_TRY_CUDA(dB.upload(b->points, s), "common");
  NAPMO_TRY_CUDA(cnt.alloc(na), "common");
  common_count<<<(int)((na + 127) / 128), 128, 0, s>>>(na, nb, dA.p, dB.p, cnt.p);
  std::vector<int> hc(na);
  NAPMO_TRY_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, na * sizeof(int), cudaMemcpyDeviceToHost, s),
                 "common");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "common");
  std::vector<long> hs(na);
  long total = 0;
  for (long i = 0; i < na; ++i) {
    hs[i] = total;
    total += hc[i];
  }
  out.assign(2 * total, 0);
  if (total == 0) return kOk;
  NAPMO_TRY_CUDA(start.upload(hs, s), "common");
  NAPMO_TRY_CUDA(pairs.alloc(2 * total), "common");
  common_write<<<(int)((na + 127) / 128), 128, 0, s>>>(na, nb, dA.p, dB.p, start.p, pairs.p);
  NAPMO_TRY_CUDA(cudaMemcpyAsync(out.data(), pairs.p, 2 * total * sizeof(int),
                                 cudaMemcpyDeviceToHost, s),
                 "common");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "common");
  return kOk;
}

}  // namespace napmo

using namespace napmo;

extern "C" {

// ------------------------------------------------------------ SCF step
void wavefunction_guess_hcore(WaveFunction *psi) {
  guarded([&] { return diag_and_density(psi, psi->H, true, nullptr, false); });
}

void wavefunction_compute_coefficients(WaveFunction *psi) {
  guarded([&] { return diag_and_density(psi, psi->F, false, nullptr, false); });
}

// L = D; solve F C = S C e; D = eta C_occ C_occ^T; energy and rmsd.
void wavefunction_iterate(WaveFunction *psi) {
  guarded([&] {
    const size_t nn = (size_t)psi->ndim * psi->ndim;
    for (size_t i = 0; i < nn; ++i) psi->L[i] = psi->D[i];
    double er[2] = {0.0, 0.0};
    int st = diag_and_density(psi, psi->F, true, er, true);
    if (st) return st;
    psi->energy = er[0] + psi->xc_energy;
    psi->rmsd = sqrt(er[1]);
    return kOk;
  });
}

void wavefunction_compute_density(WaveFunction *psi) {
  guarded([&] {
    cudaStream_t s = host_api_stream();
    const int n = psi->ndim;
    const size_t nn = (size_t)n * n;
    for (size_t i = 0; i < nn; ++i) psi->L[i] = psi->D[i];
    DevBuf<double> C, D, L, Z, out;
    NAPMO_TRY_CUDA(C.upload(psi->C, nn, s), "upload");
    NAPMO_TRY_CUDA(D.alloc(nn), "alloc");
    NAPMO_TRY_CUDA(L.upload(psi->L, nn, s), "upload");
    NAPMO_TRY_CUDA(Z.alloc(nn), "alloc");
    NAPMO_TRY_CUDA(cudaMemsetAsync(Z.p, 0, nn * sizeof(double), s), "zero");
    NAPMO_TRY_CUDA(out.alloc(2), "alloc");
    density_from_c<<<(int)((nn + 255) / 256), 256, 0, s>>>(n, psi->occupation, psi->eta, C.p, D.p);
    energy_rmsd<<<1, 256, 0, s>>>(n, D.p, Z.p, Z.p, Z.p, L.p, out.p);
    double er[2];
    NAPMO_TRY_CUDA(cudaMemcpyAsync(psi->D, D.p, nn * sizeof(double), cudaMemcpyDeviceToHost, s), "D");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(er, out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s), "r");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "sync");
    psi->rmsd = sqrt(er[1]);
    return kOk;
  });
}

void wavefunction_compute_energy(WaveFunction *psi) {
  guarded([&] {
    cudaStream_t s = host_api_stream();
    const size_t nn = (size_t)psi->ndim * psi->ndim;
    DevBuf<double> D, H, G, J, out;
    NAPMO_TRY_CUDA(D.upload(psi->D, nn, s), "upload");
    NAPMO_TRY_CUDA(H.upload(psi->H, nn, s), "upload");
    NAPMO_TRY_CUDA(G.upload(psi->G, nn, s), "upload");
    NAPMO_TRY_CUDA(J.upload(psi->J, nn, s), "upload");
    NAPMO_TRY_CUDA(out.alloc(2), "alloc");
    energy_rmsd<<<1, 256, 0, s>>>(psi->ndim, D.p, H.p, G.p, J.p, nullptr, out.p);
    double er[2];
    NAPMO_TRY_CUDA(cudaMemcpyAsync(er, out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s), "e");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "sync");
    psi->energy = er[0] + psi->xc_energy;
    return kOk;
  });
}

// X(i,j) /= sqrt(O(j)); X = X * V^T with V the incoming X (src/wavefunction/
// wavefunction.cpp:40-62).  Set-up only (once per basis).
void wavefunction_transformation_matrix(WaveFunction *psi) {
  const int n = psi->ndim;
  std::vector<double> V(psi->X, psi->X + (size_t)n * n), Y((size_t)n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) Y[(size_t)i * n + j] = V[(size_t)i * n + j] / sqrt(psi->O[j]);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double acc = 0.0;
      for (int k = 0; k < n; ++k) acc += Y[(size_t)i * n + k] * V[(size_t)j * n + k];
      psi->X[(size_t)i * n + j] = acc;
    }
}

// ------------------------------------------------------------ MultiGrid
MultiGrid *MultiGrid_new(int ns) {
  auto *m = new MultiGrid;
  m->nspecies = ns;
  return m;
}
void MultiGrid_del(MultiGrid *m) { delete m; }
int MultiGrid_add_grid(MultiGrid *m, BeckeGrid *g) {
  m->grids.push_back(g);
  return (int)m->grids.size() - 1;
}
int MultiGrid_get_ngrids(MultiGrid *m) { return (int)m->grids.size(); }
int MultiGrid_get_nspecies(MultiGrid *m) { return m->nspecies; }
int *MultiGrid_get_common_index(MultiGrid *m, int a, int b) {
  int *result = nullptr;
  guarded([&] {
    auto key = std::make_pair(std::min(a, b), std::max(a, b));
    auto it = m->index.find(key);
    if (it == m->index.end()) {
      std::vector<int> v;
      int st = common_points(m->grids[a], m->grids[b], v);
      if (st) return st;
      it = m->index.emplace(key, std::move(v)).first;
    }
    result = it->second.data();
    return kOk;
  });
  return result;
}
int MultiGrid_get_common_index_size(MultiGrid *m, int a, int b) {
  auto it = m->index.find(std::make_pair(std::min(a, b), std::max(a, b)));
  return it == m->index.end() ? -1 : (int)it->second.size() / 2;
}

// ------------------------------------------- out-of-path stubs (libint etc.)
#define NAPMO_STUB(ret, name, args, val)                                          \
  ret name args {                                                                 \
    set_error(kNotSupported, #name ": analytic libint integrals are not part of " \
                                   "the grid-quadrature path");                   \
    return val;                                                                   \
  }
NAPMO_STUB(void, LibintInterface_init_2body_ints, (void *), )
NAPMO_STUB(void *, LibintInterface_compute_2body_ints, (void *, double *), nullptr)
NAPMO_STUB(void, LibintInterface_compute_2body_direct, (void *, double *, double *), )
NAPMO_STUB(void, LibintInterface_compute_coupling_direct, (void *, void *, double *, double *), )
NAPMO_STUB(void *, LibintInterface_diis_new, (int), nullptr)
NAPMO_STUB(void, LibintInterface_diis, (void *, void *), )
NAPMO_STUB(void, wavefunction_compute_2body_matrix, (WaveFunction *, void *), )
#undef NAPMO_STUB

void *AuxiliaryBasis_new(void *) {
  set_error(kNotSupported, "the auxiliary Slater basis is not part of the grid-quadrature path");
  return nullptr;
}
void AuxiliaryBasis_del(void *) {}
double *AuxiliaryBasis_get_aobasis(void *) { return nullptr; }
int AuxiliaryBasis_get_nao(void *) { return 0; }

}  // extern "C"
