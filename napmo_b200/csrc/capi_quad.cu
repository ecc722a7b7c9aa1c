// C-ABI of the grid quadratures: nAPMO's nwavefunction_* entry points
// (src/wavefunction/nwavefunction.cpp, bound in napmo/__init__.py:177-191),
// the device-pointer twins napmo_gpu_density / napmo_gpu_quadrature, and the
// Fock-build plan that keeps phi, the grid and the Poisson tables resident in
// HBM across SCF iterations.
#include <algorithm>
#include <cstdint>
#include <atomic>
#include <memory>
#include <vector>

#include "capi_common.cuh"
#include "host.h"
#include "kernels.cuh"
#include "wavefunction.h"

namespace napmo {

struct PoissonPlan;
int grid_poisson_plan(BeckeGrid *g, int lmax, cudaStream_t s, PoissonPlan **out);
int run_poisson(BeckeGrid *g, PoissonPlan *p, const double *rho_dev, double *v_dev,
                bool accumulate, cudaStream_t s, double tol, const int *keep,
                unsigned long long key);
int run_poisson_many(BeckeGrid *g, PoissonPlan *p, int k, const double *rho_dev, long ld,
                     double *v_dev, cudaStream_t s, double tol, const int *keep,
                     unsigned long long key);

// Truncation tolerance (a.u.) of the Poisson potential evaluation that
// precision 1 selects: each (atom, radial interval) drops l-blocks whose
// bounded contribution sums to at most this, so every point's potential moves
// by at most natom x 1e-9.  Measured at C20H42 (62 atoms, int8 build against
// the untruncated FP64 one): energy error 2.45e-8 Eh at 1e-10, 2.95e-8 at
// 1e-9, 8.1e-8 at 1e-8, 1.0e-6 at 1e-7 -- 1e-9 keeps a factor 30 inside the
// mode's 1e-6 Eh budget.
constexpr double kMixedPoissonTol = 1e-9;

// Point screening of precision 1: points with |wb w| max_mu phi_mu(p)^2 below
// this carry no weight that matters (each changes an element of F by at most
// 1e-24 |v(p)|); about a fifth of a Becke grid's points (the outer radial
// shells and points deep in other atoms' cells), skipped by the density, the
// quadrature and the potential evaluation.
constexpr double kMixedScreenTol = 1e-24;
int basis_device(BasisSet *b, cudaStream_t s, const DeviceBasis **out);

// ---------------------------------------------------------------- helpers
// Host phi [n][npoint] -> device [n][ld] with ld = padded, zero pad columns.
static int upload_phi(const double *phi, int n, int npoint, long ld, DevBuf<double> &d,
                      cudaStream_t s) {
  NAPMO_TRY_CUDA(d.alloc((size_t)n * ld), "alloc phi");
  NAPMO_TRY_CUDA(cudaMemsetAsync(d.p, 0, (size_t)n * ld * sizeof(double), s), "phi");
  NAPMO_TRY_CUDA(cudaMemcpy2DAsync(d.p, ld * sizeof(double), phi, npoint * sizeof(double),
                                   npoint * sizeof(double), n, cudaMemcpyHostToDevice, s),
                 "upload phi");
  return kOk;
}

// F = A diag(wb w v) B^T on the device from host operands (B = A if null).
static int host_quadrature(BeckeGrid *g, int n, const double *A, const double *B,
                           const double *v, double *F) {
  cudaStream_t s = host_api_stream();
  const int N = g->size;
  const long ld = padded_points(N);
  DevBuf<double> dA, dB, dv, wv, dF, work;
  int st = upload_phi(A, n, N, ld, dA, s);
  if (st) return st;
  if (B) {
    st = upload_phi(B, n, N, ld, dB, s);
    if (st) return st;
  }
  NAPMO_TRY_CUDA(dv.upload(v, N, s), "upload potential");
  NAPMO_TRY_CUDA(wv.alloc(ld), "alloc");
  NAPMO_TRY_CUDA(cudaMemsetAsync(wv.p, 0, ld * sizeof(double), s), "wv");
  NAPMO_TRY_CUDA(launch_combine_weights(N, g->dev.wb, g->dev.w, 1.0, dv.p, nullptr, wv.p, s),
                 "weights");
  NAPMO_TRY_CUDA(dF.alloc((size_t)n * n), "alloc");
  NAPMO_TRY_CUDA(work.alloc(quadrature_workspace_bytes(n, N) / sizeof(double) + 1), "alloc");
  NAPMO_TRY_CUDA(launch_quadrature_f64(n, N, dA.p, ld, wv.p, dF.p, work.p, s,
                                       B ? dB.p : nullptr),
                 "quadrature");
  NAPMO_TRY_CUDA(cudaMemcpyAsync(F, dF.p, (size_t)n * n * sizeof(double),
                                 cudaMemcpyDeviceToHost, s),
                 "download");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "sync");
  return kOk;
}

// ------------------------------------------------------------- Fock plan
struct FockPlan {
  BeckeGrid *grid = nullptr;
  BasisSet *basis = nullptr;
  int n = 0, lmax = 0;
  int mode = 0;  // 0 FP64, 1 int8 slices on the tensor cores
  double poisson_tol = 0.0;  // truncation tolerance of the potential evaluation
  unsigned generation = 0;   // bumped by every change that captured builds depend on
  long ld = 0;
  DevBuf<double> phi, rho, v, wv, work, D, F, vext;
  Int8Plan *i8 = nullptr;
  // FP64 point screening (napmo_fock_plan_set_fp64_screening): keep flags,
  // the 16-point blocks (quadrature) and 128-point groups (density) holding a
  // kept point; key names the flags for the Poisson solve's screened lists
  double fp64_screen = 0.0;
  DevBuf<int> keep64, blocks64, groups64;
  int nblocks64 = 0, ngroups64 = 0;
  unsigned long long keep64_key = 0;
  ~FockPlan() {
    if (i8) int8_plan_destroy(i8);
  }
};

// phi of the plan's basis on its grid, evaluated again when it was released
// (napmo_fock_plan_release_phi); allocates, so it runs outside captures (the
// batches' eager warm-up builds reach it first).
static int ensure_phi(FockPlan *p, cudaStream_t s) {
  if (p->phi.p) return kOk;
  const DeviceBasis *db = nullptr;
  int e = basis_device(p->basis, s, &db);
  if (e) return e;
  BeckeGrid *g = p->grid;
  NAPMO_TRY_CUDA(p->phi.alloc((size_t)p->n * p->ld), "alloc phi");
  NAPMO_TRY_CUDA(cudaMemsetAsync(p->phi.p, 0, p->phi.n * sizeof(double), s), "phi");
  NAPMO_TRY_CUDA(launch_basis_values(*db, g->size, g->dev.x, g->dev.y, g->dev.z, p->phi.p,
                                     p->ld, nullptr, s),
                 "basis");
  return kOk;
}

// rho = density of D, in the plan's precision.
int plan_density(FockPlan *p, const double *D, double *rho, cudaStream_t s) {
  if (p->mode == 1) return int8_density(p->i8, D, rho, s);
  if (int e = ensure_phi(p, s)) return e;
  const bool scr = p->fp64_screen > 0.0;
  NAPMO_TRY_CUDA(launch_density_f64(p->n, p->grid->size, p->phi.p, p->ld, D, rho, s,
                                    scr ? p->groups64.p : nullptr, p->ngroups64,
                                    scr ? p->keep64.p : nullptr),
                 "density");
  return kOk;
}

// F = phi diag(p->wv) phi^T, in the plan's precision.
int plan_quadrature(FockPlan *p, double *F, cudaStream_t s) {
  if (p->mode == 1) return int8_quadrature(p->i8, p->phi.p, p->wv.p, F, s);
  if (int e = ensure_phi(p, s)) return e;
  const bool scr = p->fp64_screen > 0.0;
  NAPMO_TRY_CUDA(launch_quadrature_f64(p->n, p->grid->size, p->phi.p, p->ld, p->wv.p, F,
                                       p->work.p, s, nullptr, scr ? p->blocks64.p : nullptr,
                                       p->nblocks64),
                 "quadrature");
  return kOk;
}

// Screening flags of the plan's grid points: precision 1 always screens, FP64
// when napmo_fock_plan_set_fp64_screening enabled it (null otherwise).
const int *plan_keep(const FockPlan *p) {
  if (p->mode == 1) return p->i8 ? int8_plan_keep(p->i8) : nullptr;
  return p->fp64_screen > 0.0 ? p->keep64.p : nullptr;
}
static unsigned long long plan_keep_key(const FockPlan *p) {
  if (p->mode == 1) return p->i8 ? int8_plan_serial(p->i8) : 0;
  return p->fp64_screen > 0.0 ? p->keep64_key : 0;
}

// FP64 screening of the plan's current phi: flags, then the block and group
// lists (read back once; synchronises).
static int build_fp64_screening(FockPlan *p, double tol, cudaStream_t s) {
  if (int e = ensure_phi(p, s)) return e;
  BeckeGrid *g = p->grid;
  const int N = g->size, nb = (N + 15) / 16, ng = (N + 127) / 128;
  DevBuf<int> bf, gf;
  NAPMO_TRY_CUDA(p->keep64.alloc(N), "alloc screening");
  NAPMO_TRY_CUDA(bf.alloc(nb), "alloc screening");
  NAPMO_TRY_CUDA(gf.alloc(ng), "alloc screening");
  NAPMO_TRY_CUDA(launch_fp64_screening(p->n, N, p->phi.p, p->ld, g->dev.wb, g->dev.w, tol,
                                       p->keep64.p, bf.p, gf.p, s),
                 "screening");
  std::vector<int> hb(nb), hg(ng), lb, lg;
  NAPMO_TRY_CUDA(cudaMemcpyAsync(hb.data(), bf.p, nb * sizeof(int), cudaMemcpyDeviceToHost, s),
                 "screening");
  NAPMO_TRY_CUDA(cudaMemcpyAsync(hg.data(), gf.p, ng * sizeof(int), cudaMemcpyDeviceToHost, s),
                 "screening");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "screening");
  for (int i = 0; i < nb; ++i)
    if (hb[i]) lb.push_back(i);
  for (int i = 0; i < ng; ++i)
    if (hg[i]) lg.push_back(i);
  NAPMO_TRY_CUDA(lb.empty() ? p->blocks64.alloc(1) : p->blocks64.upload(lb, s), "screening");
  NAPMO_TRY_CUDA(lg.empty() ? p->groups64.alloc(1) : p->groups64.upload(lg, s), "screening");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "screening");
  p->nblocks64 = (int)lb.size();
  p->ngroups64 = (int)lg.size();
  // a key no other flags share (the int8 plans count from 1 upwards)
  static std::atomic<unsigned long long> next{1};
  p->keep64_key = (1ull << 63) | next++;
  p->fp64_screen = tol;
  return kOk;
}

// The build chain of napmo_fock_plan_build (stream-ordered, no host
// synchronisation, no allocation once the grid's Poisson plan exists).
int fock_build(FockPlan *p, const double *D_dev, double q, const double *vext_dev, double *F_dev,
               double *rho_out, double *v_out, cudaStream_t s) {
  BeckeGrid *g = p->grid;
  double *rho = rho_out ? rho_out : p->rho.p;
  double *v = v_out ? v_out : p->v.p;
  int e = plan_density(p, D_dev, rho, s);
  if (e) return e;
  PoissonPlan *pp = nullptr;
  e = grid_poisson_plan(g, p->lmax, s, &pp);
  if (e) return e;
  e = run_poisson(g, pp, rho, v, false, s, p->poisson_tol, plan_keep(p), plan_keep_key(p));
  if (e) return e;
  NAPMO_TRY_CUDA(launch_combine_weights(g->size, g->dev.wb, g->dev.w, q, v, vext_dev, p->wv.p, s),
                 "weights");
  return plan_quadrature(p, F_dev, s);
}

// ------------------------------------------------------------ stage batches
// A batch of FP64 Fock builds run as one launch per stage for all molecules:
// the density of every molecule by one persistent launch over (molecule,
// 128-point group) items, the Poisson solves of every molecule by one plan
// over the concatenated grids (grid_concat: each atom pairs with its own
// molecule's points), the weights by one launch, the quadratures by one
// persistent launch over (molecule, tile, chunk) items and one reduction.
// The persistent launches take their items from device work queues posted
// when the batch is set up.  Each molecule's arithmetic is that of its own
// plan, so a stage build equals the molecules' own builds bit for bit.
int grid_concat(const std::vector<BeckeGrid *> &grids, const std::vector<int> &lmax,
                cudaStream_t s, BeckeGrid **out, std::vector<int> *off);
void grid_free(BeckeGrid *g);

struct StageBatch {
  std::vector<FockPlan *> plans;
  BeckeGrid *cat = nullptr;          // the molecules' grids as one (Poisson)
  std::vector<int> off, offp;        // point offsets: unpadded, padded to 128
  DevBuf<double> rho, v, wv;         // concatenated
  DevBuf<int> keep;                  // concatenated screening flags (screened plans)
  unsigned long long keep_key = 0;
  DevBuf<DensBatchArg> dargs;
  DevBuf<QuadBatchArg> qargs;
  DevBuf<WeightBatchArg> wargs;
  DevBuf<int4> ditems, qitems;
  DevBuf<int> head, posted, status;  // [2]: density and quadrature queues
  int nd = 0, nq = 0, grid_d = 0, grid_q = 0;
  double q = 1.0, tol = 0.0;
  unsigned long long timeout_ns = 1000000000ull;
  int mode = 0;                      // the plans' precision
  Int8Batch *i8 = nullptr;           // mode 1: the int8 stages' tables
  ~StageBatch() {
    if (cat) grid_free(cat);
    if (i8) int8_batch_free(i8);
  }
};

static int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// Set-up (synchronises): the concatenated grid and its Poisson plan, the
// batch buffers, the per-molecule argument tables and the posted work queues.
int stage_batch_new(const std::vector<FockPlan *> &plans, const std::vector<double *> &D,
                    const std::vector<double *> &F, double q, cudaStream_t s, StageBatch **out) {
  std::unique_ptr<StageBatch> b(new StageBatch);
  b->plans = plans;
  b->q = q;
  const int nmol = (int)plans.size();
  std::vector<BeckeGrid *> grids;
  std::vector<int> lmax;
  b->mode = plans[0]->mode;
  for (FockPlan *p : plans) {
    if (p->mode == 0)
      if (int e = ensure_phi(p, s)) return e;
    if (p->mode != b->mode)
      return set_error(kInvalidArgument, "plans of a stage batch share one precision");
    if (p->mode == 1 && !p->i8) return set_error(kInvalidArgument, "int8 plan without images");
    if (p->lmax < 0 && p->lmax != kLmaxPerAtom)
      return set_error(kInvalidArgument, "plan without Poisson tables");
    if (p->poisson_tol != plans[0]->poisson_tol)
      return set_error(kInvalidArgument, "plans of a stage batch share one Poisson tolerance");
    grids.push_back(p->grid);
    lmax.push_back(p->lmax);
  }
  b->tol = plans[0]->poisson_tol;
  int st = grid_concat(grids, lmax, s, &b->cat, &b->off);
  if (st) return st;
  b->offp.assign(1, 0);
  for (FockPlan *p : plans) b->offp.push_back(b->offp.back() + (int)p->ld);
  NAPMO_TRY_CUDA(b->rho.alloc(std::max(b->off.back(), 1)), "alloc batch");
  NAPMO_TRY_CUDA(b->v.alloc(std::max(b->off.back(), 1)), "alloc batch");
  NAPMO_TRY_CUDA(b->wv.alloc(std::max(b->offp.back(), 1)), "alloc batch");
  bool screened = false;
  for (FockPlan *p : plans) screened = screened || plan_keep(p) != nullptr;
  if (screened) {
    NAPMO_TRY_CUDA(b->keep.alloc(std::max(b->off.back(), 1)), "alloc batch");
    for (int m = 0; m < nmol; ++m) {
      FockPlan *p = plans[m];
      int *dst = b->keep.p + b->off[m];
      if (const int *k = plan_keep(p)) {
        NAPMO_TRY_CUDA(cudaMemcpyAsync(dst, k, (size_t)p->grid->size * sizeof(int),
                                       cudaMemcpyDeviceToDevice, s),
                       "batch flags");
      } else {
        std::vector<int> ones(p->grid->size, 1);
        NAPMO_TRY_CUDA(cudaMemcpyAsync(dst, ones.data(), ones.size() * sizeof(int),
                                       cudaMemcpyHostToDevice, s),
                       "batch flags");
        NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch flags");
      }
    }
    static std::atomic<unsigned long long> next{1};
    b->keep_key = (3ull << 62) | next++;
  }
  std::vector<DensBatchArg> da(nmol);
  std::vector<QuadBatchArg> qa(nmol);
  std::vector<WeightBatchArg> wa(nmol);
  std::vector<int4> di, qi;
  for (int m = 0; m < nmol; ++m) {
    FockPlan *p = plans[m];
    const int N = p->grid->size;
    const bool scr = p->fp64_screen > 0.0;
    da[m] = DensBatchArg{p->phi.p, p->ld, D[m], b->rho.p + b->off[m],
                         scr ? p->keep64.p : nullptr, p->n, N,
                         (p->n % 2 == 0 && reinterpret_cast<uintptr_t>(D[m]) % 16 == 0) ? 1 : 0,
                         0};
    std::vector<int> groups, blocks;
    if (scr) {
      groups.resize(p->ngroups64);
      blocks.resize(p->nblocks64);
      if (!groups.empty())
        NAPMO_TRY_CUDA(cudaMemcpy(groups.data(), p->groups64.p, groups.size() * sizeof(int),
                                  cudaMemcpyDeviceToHost),
                       "batch groups");
    } else {
      for (int gi = 0; gi < (N + 127) / 128; ++gi) groups.push_back(gi);
    }
    for (int gi : groups) di.push_back(make_int4(m, gi, 0, 0));
    const int npad = scr ? p->nblocks64 * 16 : (int)padded_points(N);
    int chunk = 0;
    const int nchunk =
        npad > 0 ? quadrature_chunking(p->n, npad, &chunk, (int)padded_points(N)) : 0;
    const int nblk = (p->n + 127) / 128, ntile = nblk * (nblk + 1) / 2;
    qa[m] = QuadBatchArg{p->phi.p, p->ld, b->wv.p + b->offp[m], p->work.p, F[m],
                         scr ? p->blocks64.p : nullptr, p->n, npad, nblk, chunk, nchunk};
    for (int c = 0; c < nchunk; ++c)
      for (int t = 0; t < ntile; ++t) qi.push_back(make_int4(m, t, c, 0));
    wa[m] = WeightBatchArg{p->grid->dev.wb, p->grid->dev.w, b->v.p + b->off[m],
                           b->wv.p + b->offp[m], N, (int)p->ld};
  }
  if (b->mode == 1) {
    std::vector<Int8Plan *> ip;
    std::vector<const double *> cD, cwv;
    std::vector<double *> rho;
    for (int m = 0; m < nmol; ++m) {
      ip.push_back(plans[m]->i8);
      cD.push_back(D[m]);
      rho.push_back(b->rho.p + b->off[m]);
      cwv.push_back(b->wv.p + b->offp[m]);
    }
    st = int8_batch_new(ip, cD, rho, cwv, F, s, &b->i8);
    if (st) return st;
  }
  NAPMO_TRY_CUDA(b->dargs.upload(da, s), "batch tables");
  NAPMO_TRY_CUDA(b->qargs.upload(qa, s), "batch tables");
  NAPMO_TRY_CUDA(b->wargs.upload(wa, s), "batch tables");
  NAPMO_TRY_CUDA(di.empty() ? b->ditems.alloc(1) : b->ditems.upload(di, s), "batch items");
  NAPMO_TRY_CUDA(qi.empty() ? b->qitems.alloc(1) : b->qitems.upload(qi, s), "batch items");
  b->nd = (int)di.size();
  b->nq = (int)qi.size();
  const int sms = sm_count();
  b->grid_d = std::max(1, std::min(b->nd, sms));
  b->grid_q = std::max(1, std::min(b->nq, sms));
  NAPMO_TRY_CUDA(b->head.alloc(2), "batch queue");
  NAPMO_TRY_CUDA(b->status.alloc(1), "batch queue");
  NAPMO_TRY_CUDA(b->posted.upload(std::vector<int>{b->nd, b->nq}, s), "batch queue");
  NAPMO_TRY_CUDA(cudaMemsetAsync(b->status.p, 0, sizeof(int), s), "batch queue");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch set-up");
  *out = b.release();
  return kOk;
}

void stage_batch_free(StageBatch *b) { delete b; }

static BatchQueue stage_queue(StageBatch *b, int which) {
  return BatchQueue{which == 0 ? b->ditems.p : b->qitems.p, which == 0 ? b->nd : b->nq,
                    b->head.p + which, b->posted.p + which, b->status.p, b->timeout_ns};
}

// One build of every molecule (stream-ordered, no allocation, capturable).
int stage_batch_build(StageBatch *b, cudaStream_t s) {
  const int nmol = (int)b->plans.size();
  NAPMO_TRY_CUDA(cudaMemsetAsync(b->head.p, 0, 2 * sizeof(int), s), "batch queue");
  if (b->keep.p)  // screened plans compute only the groups holding a kept point
    NAPMO_TRY_CUDA(cudaMemsetAsync(b->rho.p, 0, (size_t)b->off.back() * sizeof(double), s),
                   "batch rho");
  if (b->mode == 1) {  // int8 slices on the tensor cores, one batched launch per stage
    int e = int8_batch_density(b->i8, s);
    if (e) return e;
    e = run_poisson(b->cat, b->cat->poisson, b->rho.p, b->v.p, false, s, b->tol, b->keep.p,
                    b->keep_key);
    if (e) return e;
    NAPMO_TRY_CUDA(launch_combine_weights_batch(b->wargs.p, nmol, b->q, s), "weights");
    return int8_batch_quadrature(b->i8, s);
  }
  NAPMO_TRY_CUDA(launch_density_batch(b->dargs.p, stage_queue(b, 0), b->grid_d, s), "density");
  int e = run_poisson(b->cat, b->cat->poisson, b->rho.p, b->v.p, false, s, b->tol,
                      b->keep.p, b->keep_key);
  if (e) return e;
  NAPMO_TRY_CUDA(launch_combine_weights_batch(b->wargs.p, nmol, b->q, s), "weights");
  NAPMO_TRY_CUDA(launch_quadrature_batch(b->qargs.p, stage_queue(b, 1), b->grid_q, s),
                 "quadrature");
  NAPMO_TRY_CUDA(launch_quadrature_reduce_batch(b->qargs.p, nmol, s), "quadrature reduce");
  return kOk;
}

// The density stage with a queue that was never posted: every CTA's wait runs
// out after timeout_ns and records kDeviceTimeout (read back into *status,
// then cleared); the batch's queues are left as they were.  Synchronises.
int stage_batch_queue_selftest(StageBatch *b, unsigned long long timeout_ns, cudaStream_t s,
                               int *status) {
  DevBuf<int> never;
  NAPMO_TRY_CUDA(never.upload(std::vector<int>{0}, s), "self-test");
  NAPMO_TRY_CUDA(cudaMemsetAsync(b->head.p, 0, 2 * sizeof(int), s), "self-test");
  NAPMO_TRY_CUDA(cudaMemsetAsync(b->status.p, 0, sizeof(int), s), "self-test");
  BatchQueue q = stage_queue(b, 0);
  q.posted = never.p;
  q.timeout_ns = timeout_ns;
  NAPMO_TRY_CUDA(launch_density_batch(b->dargs.p, q, b->grid_d, s), "self-test");
  NAPMO_TRY_CUDA(cudaMemcpyAsync(status, b->status.p, sizeof(int), cudaMemcpyDeviceToHost, s),
                 "self-test");
  NAPMO_TRY_CUDA(cudaMemsetAsync(b->status.p, 0, sizeof(int), s), "self-test");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "self-test");
  return kOk;
}

// Device error word of the batch's work queues (0 or kDeviceTimeout); clears it.
int stage_batch_status(StageBatch *b, cudaStream_t s, int *status) {
  NAPMO_TRY_CUDA(cudaMemcpyAsync(status, b->status.p, sizeof(int), cudaMemcpyDeviceToHost, s),
                 "batch status");
  NAPMO_TRY_CUDA(cudaMemsetAsync(b->status.p, 0, sizeof(int), s), "batch status");
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch status");
  return kOk;
}

int fock_plan_nbasis(const FockPlan *p) { return p->n; }
Int8Plan *fock_plan_int8(FockPlan *p) { return p->mode == 1 ? p->i8 : nullptr; }

// State a captured build depends on: the plan's own changes (precision,
// Poisson tolerance, refresh) and its grid's moves.
unsigned long long fock_plan_state(const FockPlan *p) {
  return ((unsigned long long)p->generation << 32) | p->grid->generation;
}

}  // namespace napmo

using namespace napmo;

extern "C" {

// -------------------------------------------------- nAPMO nwavefunction_*
// res = phi diag(wb w other_J) phi^T   (coupling / Coulomb-type matrix)
void nwavefunction_compute_coupling(WaveFunction *psi, BeckeGrid *grid, double *phi,
                                    double *other_J, double *res) {
  guarded([&] { return host_quadrature(grid, psi->ndim, phi, nullptr, other_J, res); });
}

// psi->XC = phi diag(wb w xc_vrho) phi^T
void nwavefunction_compute_xc_matrix(WaveFunction *psi, BeckeGrid *grid, double *phi,
                                     double *xc_vrho) {
  guarded([&] { return host_quadrature(grid, psi->ndim, phi, nullptr, xc_vrho, psi->XC); });
}

// psi->G = int phi_i phi_j J + x_factor int phi_i K_j (upper triangle mirrored)
void nwavefunction_compute_2body_matrix(WaveFunction *psi, BeckeGrid *grid, double *phi,
                                        double *J, double *K) {
  guarded([&] {
    const int n = psi->ndim;
    std::vector<double> coul((size_t)n * n), exch((size_t)n * n, 0.0);
    int st = host_quadrature(grid, n, phi, nullptr, J, coul.data());
    if (st) return st;
    if (psi->x_factor != 0.0) {
      std::vector<double> ones(grid->size, 1.0);
      st = host_quadrature(grid, n, phi, K, ones.data(), exch.data());
      if (st) return st;
    }
    for (size_t i = 0; i < (size_t)n * n; ++i) psi->G[i] = coul[i] + psi->x_factor * exch[i];
    return kOk;
  });
}

// output[p] = sum_ij dm_ij phi_i(p) phi_j(p) on every grid point.  nAPMO's
// version returns from the whole function as soon as one point is screened
// (nwavefunction.cpp:132-133); here every point is evaluated and the
// screening arguments are accepted but not needed.
void nwavefunction_compute_density_from_dm(BasisSet *basis, BeckeGrid *grid, double *dm,
                                           double *output, double epsilon, double *dmmaxrow) {
  (void)epsilon;
  (void)dmmaxrow;
  guarded([&] {
    cudaStream_t s = host_api_stream();
    const int n = (int)basis->cont.size(), N = grid->size;
    const long ld = padded_points(N);
    const DeviceBasis *db = nullptr;
    int st = basis_device(basis, s, &db);
    if (st) return st;
    DevBuf<double> phi, D, rho;
    NAPMO_TRY_CUDA(phi.alloc((size_t)n * ld), "alloc");
    NAPMO_TRY_CUDA(cudaMemsetAsync(phi.p, 0, (size_t)n * ld * sizeof(double), s), "phi");
    NAPMO_TRY_CUDA(D.upload(dm, (size_t)n * n, s), "upload dm");
    NAPMO_TRY_CUDA(rho.alloc(N), "alloc");
    NAPMO_TRY_CUDA(launch_basis_values(*db, N, grid->dev.x, grid->dev.y, grid->dev.z, phi.p,
                                       ld, nullptr, s),
                   "basis");
    NAPMO_TRY_CUDA(launch_density_f64(n, N, phi.p, ld, D.p, rho.p, s), "density");
    NAPMO_TRY_CUDA(cudaMemcpyAsync(output, rho.p, N * sizeof(double), cudaMemcpyDeviceToHost, s),
                   "download");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "sync");
    return kOk;
  });
}

// ----------------------------------------------------------- device API
// rho[p] = sum_{mu,nu} D[mu][nu] phi[mu][p] phi[nu][p]; phi [n][ld] with
// ld >= padded(npoint) and zero padding, D [n][n] symmetric.
int napmo_gpu_density(int n, int npoint, const double *phi, long ld, const double *D,
                      double *rho, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(ld >= padded_points(npoint) && ld % 2 == 0, "ld too small or odd");
    NAPMO_TRY_CUDA(launch_density_f64(n, npoint, phi, ld, D, rho, (cudaStream_t)stream),
                   "density");
    return kOk;
  });
}

// F[mu][nu] = sum_p phi[mu][p] wv[p] psi[nu][p] (psi = phi when null), upper
// triangle mirrored; wv zero padded to padded(npoint).  Scratch is taken
// from the stream-ordered allocator and released on the same stream.
int napmo_gpu_quadrature(int n, int npoint, const double *phi, const double *psi, long ld,
                         const double *wv, double *F, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(n > 0 && npoint >= 0, "n must be positive, npoint >= 0");
    NAPMO_REQUIRE(ld >= padded_points(npoint) && ld % 2 == 0, "ld too small or odd");
    cudaStream_t s = (cudaStream_t)stream;
    if (npoint == 0) {  // empty grid: F = 0
      NAPMO_TRY_CUDA(cudaMemsetAsync(F, 0, (size_t)n * n * sizeof(double), s), "F");
      return kOk;
    }
    void *work = nullptr;
    const size_t bytes = quadrature_workspace_bytes(n, npoint);
    NAPMO_TRY_CUDA(cudaMallocAsync(&work, bytes, s), "quadrature workspace");
    cudaError_t e = launch_quadrature_f64(n, npoint, phi, ld, wv, F, (double *)work, s, psi);
    cudaFreeAsync(work, s);
    NAPMO_TRY_CUDA(e, "quadrature");
    return kOk;
  });
}

// wv[p] = wb[p] w[p] (q v[p] + vext[p]) (either potential may be null);
// entries npoint..padded(npoint) are zeroed.
int napmo_gpu_combine_weights(int npoint, const double *wb, const double *w, double q,
                              const double *v, const double *vext, double *wv, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    const long pad = padded_points(npoint);
    if (pad > npoint)
      NAPMO_TRY_CUDA(cudaMemsetAsync(wv + npoint, 0, (pad - npoint) * sizeof(double), s), "wv");
    NAPMO_TRY_CUDA(launch_combine_weights(npoint, wb, w, q, v, vext, wv, s), "weights");
    return kOk;
  });
}

// ------------------------------------------------------------- Fock plan
// A Fock-build plan evaluates phi for `basis` on `grid` once and keeps it,
// the grid mirror and the Poisson tables (for `lmax`) resident on the device.
FockPlan *napmo_fock_plan_new(BeckeGrid *grid, BasisSet *basis, int lmax, void *stream) {
  FockPlan *p = nullptr;
  int st = guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    p = new FockPlan;
    p->grid = grid;
    p->basis = basis;
    p->n = (int)basis->cont.size();
    p->lmax = lmax;
    p->ld = padded_points(grid->size);
    const DeviceBasis *db = nullptr;
    int e = basis_device(basis, s, &db);
    if (e) return e;
    NAPMO_TRY_CUDA(p->phi.alloc((size_t)p->n * p->ld), "alloc phi");
    NAPMO_TRY_CUDA(cudaMemsetAsync(p->phi.p, 0, p->phi.n * sizeof(double), s), "phi");
    NAPMO_TRY_CUDA(launch_basis_values(*db, grid->size, grid->dev.x, grid->dev.y, grid->dev.z,
                                       p->phi.p, p->ld, nullptr, s),
                   "basis");
    NAPMO_TRY_CUDA(p->rho.alloc(p->ld), "alloc");
    NAPMO_TRY_CUDA(p->v.alloc(p->ld), "alloc");
    NAPMO_TRY_CUDA(p->wv.alloc(p->ld), "alloc");
    NAPMO_TRY_CUDA(cudaMemsetAsync(p->wv.p, 0, p->ld * sizeof(double), s), "wv");
    NAPMO_TRY_CUDA(p->work.alloc(quadrature_workspace_bytes(p->n, grid->size) / 8 + 1), "alloc");
    NAPMO_TRY_CUDA(p->D.alloc((size_t)p->n * p->n), "alloc");
    NAPMO_TRY_CUDA(p->F.alloc((size_t)p->n * p->n), "alloc");
    if (lmax >= 0 || lmax == kLmaxPerAtom) {
      PoissonPlan *pp = nullptr;
      e = grid_poisson_plan(grid, lmax, s, &pp);
      if (e) return e;
    }
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "plan");
    return kOk;
  });
  if (st) {
    delete p;
    return nullptr;
  }
  return p;
}

void napmo_fock_plan_free(FockPlan *p) { delete p; }

// After the plan's grid or basis moved (napmo_grid_set_centers,
// napmo_basis_set_origins): re-evaluates the basis on the grid into the
// plan's own buffer (no allocation) and rebuilds what derives from it (the
// int8 operand images of precision 1, the Poisson tables).  Synchronises.
int napmo_fock_plan_refresh(FockPlan *p, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    BeckeGrid *g = p->grid;
    NAPMO_REQUIRE(padded_points(g->size) == p->ld && (int)p->basis->cont.size() == p->n,
                  "plan no longer matches its grid or basis sizes");
    const DeviceBasis *db = nullptr;
    int e = basis_device(p->basis, s, &db);
    if (e) return e;
    const bool released = !p->phi.p;
    if (released) {
      e = ensure_phi(p, s);  // evaluates it at the new geometry
      if (e) return e;
    } else {
      NAPMO_TRY_CUDA(launch_basis_values(*db, g->size, g->dev.x, g->dev.y, g->dev.z, p->phi.p,
                                         p->ld, nullptr, s),
                     "basis");
    }
    if (p->lmax >= 0 || p->lmax == kLmaxPerAtom) {
      PoissonPlan *pp = nullptr;
      e = grid_poisson_plan(g, p->lmax, s, &pp);
      if (e) return e;
    }
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "refresh");
    ++p->generation;
    if (p->fp64_screen > 0.0) {
      e = build_fp64_screening(p, p->fp64_screen, s);
      if (e) return e;
    }
    if (p->i8) {
      int8_plan_destroy(p->i8);
      p->i8 = nullptr;
      cudaStream_t hs = host_api_stream();
      e = int8_plan_create(&p->i8, p->n, g->size, p->phi.p, p->ld, g->dev.wb, g->dev.w,
                           kMixedScreenTol, hs);
      if (e) return e;
      NAPMO_TRY_CUDA(cudaStreamSynchronize(hs), "int8 operand images");
    }
    if (released && p->mode == 1) p->phi.reset();  // it was released: release it again
    return kOk;
  });
}

// Frees the plan's FP64 phi while it runs in precision 1 (the int8 builds
// read only their images): n x ld doubles, 7.6 GB at C20H42.  Whatever needs
// phi again (FP64 builds, napmo_fock_plan_info, screening, a new int8 image)
// evaluates it again first.  No counterpart in nAPMO.  Synchronises.
int napmo_fock_plan_release_phi(FockPlan *p) {
  return guarded([&] {
    NAPMO_REQUIRE(p->mode == 1 && p->i8, "phi can be released in precision 1 only");
    NAPMO_TRY_CUDA(cudaDeviceSynchronize(), "sync");
    p->phi.reset();
    ++p->generation;
    return kOk;
  });
}

int napmo_fock_plan_info(FockPlan *p, int *n, int *npoint, long *ld, double **phi) {
  return guarded([&] {
    *n = p->n;
    *npoint = p->grid->size;
    *ld = p->ld;
    if (int e = ensure_phi(p, host_api_stream())) return e;
    NAPMO_TRY_CUDA(cudaStreamSynchronize(host_api_stream()), "phi");
    *phi = p->phi.p;
    return kOk;
  });
}

// rho_dev[p] = density of D_dev on the plan's grid.
int napmo_fock_plan_density(FockPlan *p, const double *D_dev, double *rho_dev, void *stream) {
  return guarded([&] {
    return plan_density(p, D_dev, rho_dev, (cudaStream_t)stream);
  });
}

// F_dev = phi diag(wb w (q v + vext)) phi^T (v, vext device, either may be null).
int napmo_fock_plan_quadrature(FockPlan *p, double q, const double *v_dev,
                               const double *vext_dev, double *F_dev, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    BeckeGrid *g = p->grid;
    NAPMO_TRY_CUDA(launch_combine_weights(g->size, g->dev.wb, g->dev.w, q, v_dev, vext_dev,
                                          p->wv.p, s),
                   "weights");
    return plan_quadrature(p, F_dev, s);
  });
}

// v (device) = V_H[rho] (device) on the plan's grid, with the plan's lmax
// and Poisson tolerance (stream-ordered).
int napmo_fock_plan_poisson(FockPlan *p, const double *rho_dev, double *v_dev, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    PoissonPlan *pp = nullptr;
    int e = grid_poisson_plan(p->grid, p->lmax, s, &pp);
    if (e) return e;
    return run_poisson(p->grid, pp, rho_dev, v_dev, false, s, p->poisson_tol, plan_keep(p),
                       plan_keep_key(p));
  });
}

// k Poisson solves on the plan's grid: v[j] = V_H[rho[j]] for device rows of
// ld >= npoint doubles (the exchange pair densities of an SCF step), in one
// call: each launch of the pipeline takes a batch of solves.
int napmo_fock_plan_poisson_many(FockPlan *p, int k, const double *rho_dev, long ld,
                                 double *v_dev, void *stream) {
  return guarded([&] {
    NAPMO_REQUIRE(k >= 0 && ld >= p->grid->size, "k < 0 or ld < grid size");
    cudaStream_t s = (cudaStream_t)stream;
    PoissonPlan *pp = nullptr;
    int e = grid_poisson_plan(p->grid, p->lmax, s, &pp);
    if (e) return e;
    return run_poisson_many(p->grid, pp, k, rho_dev, ld, v_dev, s, p->poisson_tol,
                            plan_keep(p), plan_keep_key(p));
  });
}

// One grid Fock build of a species with its own density:
//   rho = density(D), v = q * V_H[rho] (Becke-Dickson Poisson), and
//   F = phi diag(wb w (v + vext)) phi^T.
// rho_out / v_out (device, optional) receive the density and the potential.
int napmo_fock_plan_build(FockPlan *p, const double *D_dev, double q, const double *vext_dev,
                          double *F_dev, double *rho_out, double *v_out, void *stream) {
  return guarded([&] {
    return fock_build(p, D_dev, q, vext_dev, F_dev, rho_out, v_out, (cudaStream_t)stream);
  });
}

// Same build from host buffers: D_host [n][n] in, F_host [n][n] out, vext_host
// (npoint, optional).  Copies run on the given stream inside the call.
int napmo_fock_plan_build_host(FockPlan *p, const double *D_host, double q,
                               const double *vext_host, double *F_host, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nn = (size_t)p->n * p->n;
    NAPMO_TRY_CUDA(cudaMemcpyAsync(p->D.p, D_host, nn * sizeof(double), cudaMemcpyHostToDevice, s),
                   "D upload");
    const double *vext = nullptr;
    if (vext_host) {
      if (!p->vext.p) NAPMO_TRY_CUDA(p->vext.alloc(p->grid->size), "alloc");
      NAPMO_TRY_CUDA(cudaMemcpyAsync(p->vext.p, vext_host, p->grid->size * sizeof(double),
                                     cudaMemcpyHostToDevice, s),
                     "vext upload");
      vext = p->vext.p;
    }
    int e = napmo_fock_plan_build(p, p->D.p, q, vext, p->F.p, nullptr, nullptr, stream);
    if (e) return e;
    NAPMO_TRY_CUDA(cudaMemcpyAsync(F_host, p->F.p, nn * sizeof(double), cudaMemcpyDeviceToHost, s),
                   "F download");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "sync");
    return kOk;
  });
}

}  // extern "C"

namespace napmo {
namespace {
// v[p] = sum_A Z_A / |r_p - R_A|  (napmo/wavefunction/nnuclear.py:15-37)
__global__ void nuclear_potential_kernel(int npoint, const double *__restrict__ x,
                                         const double *__restrict__ y,
                                         const double *__restrict__ z, int nq,
                                         const double *__restrict__ q, double *__restrict__ v) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoint) return;
  double acc = 0.0;
  for (int a = 0; a < nq; ++a) {
    const double dx = q[4 * a] - x[p], dy = q[4 * a + 1] - y[p], dz = q[4 * a + 2] - z[p];
    acc += q[4 * a + 3] / sqrt(dx * dx + dy * dy + dz * dz);
  }
  v[p] = acc;
}
}  // namespace
}  // namespace napmo

extern "C" {
// v (device, npoint) = sum over point charges (host [nq][4] = x, y, z, Z) of
// Z / |r - R| at device points (SoA).
int napmo_gpu_nuclear_potential(int npoint, const double *x, const double *y, const double *z,
                                int nq, const double *charges, double *v, void *stream) {
  return napmo::guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    napmo::DevBuf<double> dq;
    NAPMO_TRY_CUDA(dq.upload(charges, 4 * (size_t)nq, s), "charges");
    napmo::nuclear_potential_kernel<<<(npoint + 255) / 256, 256, 0, s>>>(npoint, x, y, z, nq,
                                                                        dq.p, v);
    NAPMO_TRY_CUDA(cudaGetLastError(), "nuclear potential");
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "nuclear potential");
    return napmo::kOk;
  });
}
}  // extern "C"

// ------------------------------------------------ int8-slice tensor cores
extern "C" {

// Precision of a plan's contractions: 0 = FP64 (CUDA cores, default),
// 1 = int8 slices on the tensor cores (four balanced base-256 digits per
// value against a group exponent, exact int32 accumulation in TMEM).  The
// Poisson solve stays FP64 in both modes; mode 1 also sets the plan's Poisson
// truncation tolerance to 1e-9 a.u. (mode 0 to 0, every (l, m) evaluated).
// Switching to 1 builds phi's operand images (device-synchronous, once per
// plan); switching to 0 evaluates phi again when it was released.
int napmo_fock_plan_set_precision(FockPlan *p, int mode) {
  return napmo::guarded([&] {
    NAPMO_REQUIRE(mode == 0 || mode == 1, "precision mode must be 0 (fp64) or 1 (int8x4)");
    if (mode == 1 && !p->i8) {
      NAPMO_TRY_CUDA(cudaDeviceSynchronize(), "sync");
      cudaStream_t s = napmo::host_api_stream();
      if (int e = napmo::ensure_phi(p, s)) return e;
      BeckeGrid *g = p->grid;
      int e = napmo::int8_plan_create(&p->i8, p->n, g->size, p->phi.p, p->ld, g->dev.wb,
                                      g->dev.w, napmo::kMixedScreenTol, s);
      if (e) return e;
      NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "int8 operand images");
    }
    if (mode == 0 && !p->phi.p) {
      cudaStream_t s = napmo::host_api_stream();
      if (int e = napmo::ensure_phi(p, s)) return e;
      NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "phi");
    }
    p->mode = mode;
    p->poisson_tol = mode == 1 ? napmo::kMixedPoissonTol : 0.0;
    ++p->generation;
    return napmo::kOk;
  });
}

// Truncation tolerance (a.u., >= 0) of the plan's Poisson potential
// evaluation; napmo_fock_plan_set_precision resets it to the mode's default
// (0 for FP64, which sums every (l, m) as nAPMO does; 1e-9 for int8 slices).
int napmo_fock_plan_set_poisson_tolerance(FockPlan *p, double tol) {
  return napmo::guarded([&] {
    NAPMO_REQUIRE(tol >= 0.0 && tol < 1.0, "Poisson tolerance must be in [0, 1)");
    p->poisson_tol = tol;
    ++p->generation;
    return napmo::kOk;
  });
}

// Point screening of the FP64 mode (precision 1 always screens): tol > 0
// keeps only the points with |wb w| max_mu phi_mu(p)^2 >= tol (1e-24 is the
// int8 mode's threshold), so that the density, the potential evaluation and
// the quadrature skip the rest; 0 uses every point (nAPMO's sums).  Builds the
// flags from the plan's current phi (synchronises).
int napmo_fock_plan_set_fp64_screening(FockPlan *p, double tol, void *stream) {
  return napmo::guarded([&] {
    NAPMO_REQUIRE(tol >= 0.0 && tol < 1.0, "screening tolerance must be in [0, 1)");
    if (tol > 0.0) {
      int e = napmo::build_fp64_screening(p, tol, (cudaStream_t)stream);
      if (e) return e;
    } else {
      p->fp64_screen = 0.0;
    }
    ++p->generation;
    return napmo::kOk;
  });
}

// Point screening of the plan's current mode: *keep receives the device flags
// (one int per grid point, 1 = kept; null when every point is used) and
// *nkeep the number of kept points.
int napmo_fock_plan_screening(FockPlan *p, const int **keep, int *nkeep) {
  return napmo::guarded([&] {
    const int *k = napmo::plan_keep(p);
    *keep = k;
    int nk = p->grid->size;
    if (k && p->mode == 1) {
      nk = napmo::int8_plan_npoint(p->i8);
    } else if (k) {
      std::vector<int> h(p->grid->size);
      NAPMO_TRY_CUDA(cudaMemcpy(h.data(), k, h.size() * sizeof(int), cudaMemcpyDeviceToHost),
                     "screening flags");
      nk = 0;
      for (int x : h) nk += x;
    }
    *nkeep = nk;
    return napmo::kOk;
  });
}

// Device bytes held by the plan's int8 operand images and scratch (0 before
// precision 1 was selected).
long napmo_fock_plan_int8_bytes(FockPlan *p) {
  return p->i8 ? (long)napmo::int8_plan_device_bytes(p->i8) : 0;
}

// Device error word of the tensor-core kernels (0 = none, 5 = an mbarrier
// wait ran out); synchronises the stream.  `reset` nonzero clears it.
int napmo_tc_status(void *stream, int reset) {
  return napmo::tc_error_status((cudaStream_t)stream, reset != 0);
}

// Runs the tensor-core kernels' bounded mbarrier wait on barriers that
// nothing arrives on (about 2 s), so that the timeout path is exercised
// without a fault: out_dev[0] and [1] (device ints) receive 0 when the two
// waiting roles gave up, and napmo_tc_status then reads 5.
int napmo_tc_wait_selftest(int *out_dev, void *stream) {
  return napmo::guarded([&] { return napmo::tc_wait_selftest(out_dev, (cudaStream_t)stream); });
}

}  // extern "C"
