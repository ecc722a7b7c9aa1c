// C-ABI of the Gaussian basis side of libnapmo (PrimitiveGaussian,
// ContractedGaussian, BasisSet; nAPMO src/system/{gto,basis_set}.cpp and the
// ctypes bindings in napmo/__init__.py:197-270).  Normalisation and overlaps
// are host set-up; every evaluation on points runs in gto.cu on the GPU.
#include <vector>

#include "capi_common.cuh"
#include "host.h"
#include "kernels.cuh"

namespace napmo {

static void free_device_basis(DeviceBasis &d) {
  cudaFree(d.shell_info);
  cudaFree(d.shell_center);
  cudaFree(d.prim_zeta);
  cudaFree(d.coef);
  cudaFree(d.func_l);
  d = DeviceBasis();
}

BasisSet::~BasisSet() {
  if (dev_valid) free_device_basis(dev);
}

int upload_basis(const HostBasisPack &pk, DeviceBasis *out, cudaStream_t s) {
  DevBuf<int> info, fl;
  DevBuf<double> cen, zeta, coef;
  NAPMO_TRY_CUDA(info.upload(pk.shell_info, s), "basis upload");
  NAPMO_TRY_CUDA(cen.upload(pk.shell_center, s), "basis upload");
  NAPMO_TRY_CUDA(zeta.upload(pk.prim_zeta, s), "basis upload");
  NAPMO_TRY_CUDA(coef.upload(pk.coef, s), "basis upload");
  NAPMO_TRY_CUDA(fl.upload(pk.func_l, s), "basis upload");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "basis upload");
  out->nfunc = pk.nfunc;
  out->nshell = pk.nshell;
  out->max_nprim = pk.max_nprim;
  out->max_l = pk.max_l;
  out->shell_info = info.release();
  out->shell_center = cen.release();
  out->prim_zeta = zeta.release();
  out->coef = coef.release();
  out->func_l = fl.release();
  return kOk;
}

int basis_device(BasisSet *b, cudaStream_t s, const DeviceBasis **out) {
  if (!b->dev_valid) {
    HostBasisPack pk;
    pack_basis(b->cont, &pk);
    for (int i = 0; i < pk.nshell; ++i)
      if (pk.shell_info[6 * i + 5] > 4)
        return set_error(kNotSupported, "basis functions above L = 4 are not supported");
    int st = upload_basis(pk, &b->dev, s);
    if (st) return st;
    b->dev_valid = true;
  }
  *out = &b->dev;
  return kOk;
}

__global__ void aos_to_soa_kernel(long n, const double *__restrict__ r, double *x,
                                  double *y, double *z) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = r[3 * i];
  y[i] = r[3 * i + 1];
  z[i] = r[3 * i + 2];
}

// phi [nf][ld] (+ 3 planes of gradients) -> out [n][nf] or [n][nf][3]
__global__ void transpose_out_kernel(long n, int nf, long ld, const double *__restrict__ src,
                                     int ncomp, double *__restrict__ dst) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= n * nf * ncomp) return;
  const long p = e / (nf * ncomp);
  const int f = (int)((e / ncomp) % nf), c = (int)(e % ncomp);
  dst[e] = src[(long)c * nf * ld + (long)f * ld + p];
}

// Evaluates `cont` at host points r[n][3] into host out: values [n][nf] or
// (grad) gradients [n][nf][3].
int evaluate_on_host_points(const std::vector<ContractedGaussian> &cont, const double *r,
                            long n, double *out, bool grad) {
  cudaStream_t s = host_api_stream();
  HostBasisPack pk;
  pack_basis(cont, &pk);
  DeviceBasis db;
  int st = upload_basis(pk, &db, s);
  if (st) return st;
  struct Guard {
    DeviceBasis *d;
    ~Guard() { free_device_basis(*d); }
  } guard{&db};
  const int nf = pk.nfunc;
  const long ld = n;
  DevBuf<double> dr, x, y, z, phi, g, res;
  NAPMO_TRY_CUDA(dr.upload(r, 3 * n, s), "basis points");
  NAPMO_TRY_CUDA(x.alloc(n), "alloc");
  NAPMO_TRY_CUDA(y.alloc(n), "alloc");
  NAPMO_TRY_CUDA(z.alloc(n), "alloc");
  NAPMO_TRY_CUDA(phi.alloc((size_t)nf * ld), "alloc");
  if (grad) NAPMO_TRY_CUDA(g.alloc(3 * (size_t)nf * ld), "alloc");
  const int ncomp = grad ? 3 : 1;
  NAPMO_TRY_CUDA(res.alloc((size_t)n * nf * ncomp), "alloc");
  aos_to_soa_kernel<<<(int)((n + 255) / 256), 256, 0, s>>>(n, dr.p, x.p, y.p, z.p);
  NAPMO_TRY_CUDA(launch_basis_values(db, (int)n, x.p, y.p, z.p, phi.p, ld, g.p, s),
                 "basis kernel");
  const long total = n * nf * ncomp;
  transpose_out_kernel<<<(int)((total + 255) / 256), 256, 0, s>>>(n, nf, ld, grad ? g.p : phi.p,
                                                                  ncomp, res.p);
  NAPMO_TRY_CUDA(cudaGetLastError(), "basis transpose");
  NAPMO_TRY_CUDA(cudaMemcpyAsync(out, res.p, total * sizeof(double), cudaMemcpyDeviceToHost, s),
                 "basis download");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "basis sync");
  return kOk;
}

static ContractedGaussian single_primitive(const PrimitiveGaussian &p) {
  // a one-primitive "contraction" whose value is exactly coeff * N * poly * exp
  PrimitiveGaussian q = p;
  PrimitiveGaussian *pp = &q;
  ContractedGaussian c(&pp, 1);
  c.norma = 1.0;
  return c;
}

}  // namespace napmo

using namespace napmo;

extern "C" {

// ------------------------------------------------------------- primitive
PrimitiveGaussian *PrimitiveGaussian_new(int *ll, double *A, double z, double c) {
  return new PrimitiveGaussian(ll, A, z, c);
}
void PrimitiveGaussian_del(PrimitiveGaussian *p) { delete p; }
void PrimitiveGaussian_get_l(PrimitiveGaussian *p, int *ll) {
  for (int i = 0; i < 3; ++i) ll[i] = p->l[i];
}
void PrimitiveGaussian_get_origin(PrimitiveGaussian *p, double *A) {
  for (int i = 0; i < 3; ++i) A[i] = p->origin[i];
}
double PrimitiveGaussian_get_zeta(PrimitiveGaussian *p) { return p->zeta; }
double PrimitiveGaussian_get_coeff(PrimitiveGaussian *p) { return p->coeff; }
double PrimitiveGaussian_get_norma(PrimitiveGaussian *p) { return p->norma; }
double PrimitiveGaussian_overlap(PrimitiveGaussian *a, PrimitiveGaussian *b) {
  return overlap_primitive(*a, *b);
}
void PrimitiveGaussian_compute(PrimitiveGaussian *p, double *r, double *out, int size) {
  guarded([&] {
    std::vector<ContractedGaussian> c{single_primitive(*p)};
    return evaluate_on_host_points(c, r, size, out, false);
  });
}
void PrimitiveGaussian_deriv(PrimitiveGaussian *p, double *r, double *out, int size) {
  guarded([&] {
    std::vector<ContractedGaussian> c{single_primitive(*p)};
    return evaluate_on_host_points(c, r, size, out, true);
  });
}

// ------------------------------------------------------------ contraction
ContractedGaussian *ContractedGaussian_new(PrimitiveGaussian **p, int n) {
  return new ContractedGaussian(p, n);
}
void ContractedGaussian_del(ContractedGaussian *c) { delete c; }
int ContractedGaussian_get_nprim(ContractedGaussian *c) { return (int)c->prim.size(); }
void ContractedGaussian_get_l(ContractedGaussian *c, int *ll) {
  for (int i = 0; i < 3; ++i) ll[i] = c->l[i];
}
void ContractedGaussian_get_origin(ContractedGaussian *c, double *A) {
  for (int i = 0; i < 3; ++i) A[i] = c->origin[i];
}
double ContractedGaussian_get_norma(ContractedGaussian *c) { return c->norma; }
double ContractedGaussian_overlap(ContractedGaussian *a, ContractedGaussian *b) {
  return a->overlap(*b);
}
void ContractedGaussian_compute(ContractedGaussian *c, double *r, double *out, int size) {
  guarded([&] {
    std::vector<ContractedGaussian> v{*c};
    return evaluate_on_host_points(v, r, size, out, false);
  });
}
void ContractedGaussian_deriv(ContractedGaussian *c, double *r, double *out, int size) {
  guarded([&] {
    std::vector<ContractedGaussian> v{*c};
    return evaluate_on_host_points(v, r, size, out, true);
  });
}

// -------------------------------------------------------------- basis set
BasisSet *BasisSet_new_empty() { return new BasisSet(); }
BasisSet *BasisSet_new(ContractedGaussian **c, int n) {
  auto *b = new BasisSet();
  for (int i = 0; i < n; ++i) b->cont.push_back(*c[i]);
  for (auto &x : b->cont) {
    b->max_nprim = std::max((int)x.prim.size(), b->max_nprim);
    b->max_l = std::max(x.l[0], b->max_l);
  }
  return b;
}
void BasisSet_del(BasisSet *b) { delete b; }
void BasisSet_update(BasisSet *b, BasisSet *o) {
  b->max_nprim = std::max(b->max_nprim, o->max_nprim);
  b->max_l = std::max(b->max_l, o->max_l);
  for (auto &x : o->cont) b->cont.push_back(x);
  if (b->dev_valid) {
    free_device_basis(b->dev);
    b->dev_valid = false;
  }
}
int BasisSet_get_nbasis(BasisSet *b) { return (int)b->cont.size(); }
int BasisSet_get_max_l(BasisSet *b) { return b->max_l; }
int BasisSet_get_max_nprim(BasisSet *b) { return b->max_nprim; }

// out[n][nbasis] = phi_mu(r_p)  (GPU)
void BasisSet_compute(BasisSet *b, double *r, double *out, int size) {
  guarded([&] { return evaluate_on_host_points(b->cont, r, size, out, false); });
}
// out[n][nbasis][3] = grad phi_mu(r_p)  (GPU; analytic gradient)
void BasisSet_deriv(BasisSet *b, double *r, double *out, int size) {
  guarded([&] { return evaluate_on_host_points(b->cont, r, size, out, true); });
}

// Device API: phi[mu * ld + p] for device points (SoA); optional gradients
// grad[(c * nbasis + mu) * ld + p], c = x, y, z.
int napmo_gpu_basis_values(BasisSet *b, int npoint, const double *x, const double *y,
                           const double *z, double *phi, long ld, double *grad,
                           void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(ld >= npoint, "ld must be >= npoint");
    cudaStream_t s = (cudaStream_t)stream;
    const DeviceBasis *db = nullptr;
    int st = basis_device(b, s, &db);
    if (st) return st;
    NAPMO_TRY_CUDA(launch_basis_values(*db, npoint, x, y, z, phi, ld, grad, s), "basis kernel");
    return kOk;
  });
}

// Origins [nfunc][3] (bohr) of the basis functions, in basis order.
int napmo_basis_get_origins(BasisSet *b, double *out) {
  return guarded([&] {
    for (size_t k = 0; k < b->cont.size(); ++k)
      for (int d = 0; d < 3; ++d) out[3 * k + d] = b->cont[k].origin[d];
    return kOk;
  });
}

// Moves the basis functions to origins [nfunc][3] (bohr; the functions of one
// shell keep a common origin).  The device copy's shell centres are rewritten
// in place (no allocation); plans built on this basis re-evaluate their basis
// values with napmo_fock_plan_refresh.  No counterpart in nAPMO, which builds
// a new basis per geometry.
int napmo_basis_set_origins(BasisSet *b, const double *origins) {
  return guarded([&] {
    for (size_t k = 0; k < b->cont.size(); ++k) {
      ContractedGaussian &c = b->cont[k];
      for (int d = 0; d < 3; ++d) c.origin[d] = origins[3 * k + d];
      for (auto &pg : c.prim)
        for (int d = 0; d < 3; ++d) pg.origin[d] = origins[3 * k + d];
    }
    if (b->dev_valid) {
      HostBasisPack pk;
      pack_basis(b->cont, &pk);
      NAPMO_REQUIRE(pk.nshell == b->dev.nshell,
                    "moved functions no longer share their shell's origin");
      NAPMO_TRY_CUDA(cudaMemcpy(b->dev.shell_center, pk.shell_center.data(),
                                pk.shell_center.size() * sizeof(double), cudaMemcpyHostToDevice),
                     "move basis");
    }
    return kOk;
  });
}

// Overlap and kinetic-energy matrices (host out, [n][n] row-major) of the
// normalised contracted basis, analytic (Obara-Saika); nAPMO takes them from
// libint (libint_iface.cpp:136-190), not available here.
int napmo_basis_one_body(BasisSet *b, double *S, double *T) {
  return guarded([&] {
    one_body_matrices(b->cont, S, T);
    return kOk;
  });
}

}  // extern "C"
