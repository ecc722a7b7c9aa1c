// Batched grid Fock builds: many molecules (species) of uneven grid and basis
// sizes built by one CUDA-graph launch.
//
// The batch holds one Fock plan per molecule (napmo_fock_plan_new) and owns
// a device D and F per molecule.  On first use it runs every build once
// eagerly (lazy set-up: Poisson plans, kernel attributes, constant tables),
// then captures the builds into a graph (again after any plan changed:
// precision, Poisson tolerance, a refresh or a moved grid): the molecules are spread over
// `nstream` capture streams forked from and joined back into the batch's
// origin stream, so the graph holds nstream independent chains and small
// molecules' kernels run side by side.  A build of the whole batch is then one
// cudaGraphLaunch on the caller's stream (which may be the legacy stream).
//
// Autotuner: the launch shape of the batch is a choice of nstream and of the
// CTA budget the int8 tensor-core kernels of every molecule are sized for
// (int8_set_budget: persistent grid and split-K chunking).  napmo_fock_batch_tune
// captures the graph for each candidate (nstream in {1, 2, 4, 8, 16, 32},
// budget in {SMs, SMs/2, SMs/4, SMs/8}), times `reps` launches of each with
// CUDA events after one warm-up launch, and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "capi_common.cuh"
#include "kernels.cuh"

namespace napmo {

struct FockPlan;
int fock_build(FockPlan *p, const double *D_dev, double q, const double *vext_dev, double *F_dev,
               double *rho_out, double *v_out, cudaStream_t s);
struct StageBatch;
int stage_batch_new(const std::vector<FockPlan *> &plans, const std::vector<double *> &D,
                    const std::vector<double *> &F, double q, cudaStream_t s, StageBatch **out);
void stage_batch_free(StageBatch *b);
int stage_batch_build(StageBatch *b, cudaStream_t s);
int stage_batch_queue_selftest(StageBatch *b, unsigned long long timeout_ns, cudaStream_t s,
                               int *status);
int stage_batch_status(StageBatch *b, cudaStream_t s, int *status);
int fock_plan_nbasis(const FockPlan *p);
Int8Plan *fock_plan_int8(FockPlan *p);
unsigned long long fock_plan_state(const FockPlan *p);

struct FockBatch {
  std::vector<FockPlan *> plans;  // not owned
  std::vector<std::unique_ptr<DevBuf<double>>> D, F;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
  cudaStream_t origin = nullptr;  // capture origin (the caller's stream may be the legacy one)
  cudaGraphExec_t exec = nullptr;
  double q = 1.0;
  int nstream = 8, budget = 0;
  int mode = 0;                    // 0: per-molecule chains on streams; 1: one launch per stage
  StageBatch *stage = nullptr;     // mode 1 state (built at warm-up)
  bool warm = false;
  float tuned_ms = 0.0f;
  std::vector<unsigned long long> state;  // fock_plan_state of every plan at warm-up

  ~FockBatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (stage) stage_batch_free(stage);
    for (auto s : streams) cudaStreamDestroy(s);
    for (auto e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (origin) cudaStreamDestroy(origin);
  }
};

namespace {

constexpr int kMaxStreams = 32;

int set_budgets(FockBatch *b, int budget) {
  for (auto *p : b->plans)
    if (Int8Plan *i8 = fock_plan_int8(p)) {
      const int e = int8_set_budget(i8, budget);
      if (e) return e;
    }
  b->budget = budget;
  return kOk;
}

// True when a plan changed since the warm-up (precision, tolerance, refresh,
// moved grid): the captured graph would run on freed or stale state.
bool stale(const FockBatch *b) {
  if (b->state.size() != b->plans.size()) return true;
  for (size_t i = 0; i < b->plans.size(); ++i)
    if (fock_plan_state(b->plans[i]) != b->state[i]) return true;
  return false;
}

// Every build once, outside any capture (creates the lazily built state).
int warm_up(FockBatch *b, cudaStream_t s) {
  if (b->exec) {  // captured against the previous state
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  for (size_t i = 0; i < b->plans.size(); ++i) {
    const int e = fock_build(b->plans[i], b->D[i]->p, b->q, nullptr, b->F[i]->p, nullptr,
                             nullptr, s);
    if (e) return e;
  }
  NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch warm-up");
  if (b->stage) {
    stage_batch_free(b->stage);
    b->stage = nullptr;
  }
  if (b->mode == 1) {
    std::vector<double *> D, F;
    for (size_t i = 0; i < b->plans.size(); ++i) {
      D.push_back(b->D[i]->p);
      F.push_back(b->F[i]->p);
    }
    const int e = stage_batch_new(b->plans, D, F, b->q, s, &b->stage);
    if (e) return e;
    const int e2 = stage_batch_build(b->stage, s);  // lazily built state, outside capture
    if (e2) return e2;
    NAPMO_TRY_CUDA(cudaStreamSynchronize(s), "batch warm-up");
  }
  b->state.clear();
  for (auto *p : b->plans) b->state.push_back(fock_plan_state(p));
  b->warm = true;
  return kOk;
}

// Captures the batch with the current nstream / budget into b->exec (on the
// batch's own origin stream; the graph is launched on the caller's stream).
int capture(FockBatch *b) {
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  cudaStream_t s = b->origin;
  const int nplan = (int)b->plans.size();
  const int ns = std::max(1, std::min(b->nstream, nplan));
  if (b->mode == 1) {  // one launch per stage, all on the origin stream
    NAPMO_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "begin capture");
    const int st = stage_batch_build(b->stage, s);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &graph);
    if (st != kOk || ee != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return st != kOk ? st : cuda_status(ee, "batch capture");
    }
    const cudaError_t ce = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    NAPMO_TRY_CUDA(ce, "batch graph instantiate");
    return kOk;
  }
  NAPMO_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "begin capture");
  int st = kOk;
  cudaError_t ce = cudaEventRecord(b->fork, s);
  for (int k = 0; k < ns && ce == cudaSuccess; ++k) ce = cudaStreamWaitEvent(b->streams[k], b->fork, 0);
  for (int i = 0; i < nplan && ce == cudaSuccess && st == kOk; ++i)
    st = fock_build(b->plans[i], b->D[i]->p, b->q, nullptr, b->F[i]->p, nullptr, nullptr,
                    b->streams[i % ns]);
  for (int k = 0; k < ns && ce == cudaSuccess; ++k) {
    ce = cudaEventRecord(b->joins[k], b->streams[k]);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s, b->joins[k], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(s, &graph);
  if (st != kOk || ce != cudaSuccess || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (st != kOk) return st;
    return cuda_status(ce != cudaSuccess ? ce : ee, "batch capture");
  }
  ce = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  NAPMO_TRY_CUDA(ce, "batch graph instantiate");
  return kOk;
}

}  // namespace
}  // namespace napmo

using namespace napmo;

extern "C" {

// Batch of Fock plans (array of napmo_fock_plan_new handles, not owned; they
// must outlive the batch).  Every build uses charge q and no external
// potential; inputs and outputs are the batch's own D and F buffers.
FockBatch *napmo_fock_batch_new(void **plans, int nplan, double q) {
  FockBatch *b = nullptr;
  const int st = guarded([&] {
    NAPMO_REQUIRE(nplan >= 1, "empty batch");
    std::unique_ptr<FockBatch> bb(new FockBatch);
    bb->q = q;
    for (int i = 0; i < nplan; ++i) {
      NAPMO_REQUIRE(plans[i] != nullptr, "null plan in batch");
      auto *p = (FockPlan *)plans[i];
      const size_t nn = (size_t)fock_plan_nbasis(p) * fock_plan_nbasis(p);
      bb->plans.push_back(p);
      bb->D.emplace_back(new DevBuf<double>);
      bb->F.emplace_back(new DevBuf<double>);
      NAPMO_TRY_CUDA(bb->D.back()->alloc(nn), "alloc batch D");
      NAPMO_TRY_CUDA(bb->F.back()->alloc(nn), "alloc batch F");
      NAPMO_TRY_CUDA(cudaMemset(bb->D.back()->p, 0, nn * sizeof(double)), "zero batch D");
    }
    for (int k = 0; k < kMaxStreams; ++k) {
      cudaStream_t s;
      cudaEvent_t e;
      NAPMO_TRY_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "batch streams");
      bb->streams.push_back(s);
      NAPMO_TRY_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch events");
      bb->joins.push_back(e);
    }
    NAPMO_TRY_CUDA(cudaEventCreateWithFlags(&bb->fork, cudaEventDisableTiming), "batch events");
    NAPMO_TRY_CUDA(cudaStreamCreateWithFlags(&bb->origin, cudaStreamNonBlocking), "batch streams");
    b = bb.release();
    return kOk;
  });
  return st ? nullptr : b;
}

void napmo_fock_batch_free(FockBatch *b) { delete b; }

// Device D and F of molecule i ([n][n] row-major).
int napmo_fock_batch_buffers(FockBatch *b, int i, double **D, double **F) {
  return guarded([&] {
    NAPMO_REQUIRE(i >= 0 && i < (int)b->plans.size(), "molecule index out of range");
    *D = b->D[i]->p;
    *F = b->F[i]->p;
    return kOk;
  });
}

// All builds of the batch: one graph launch on `stream` (captured on first use).
int napmo_fock_batch_build(FockBatch *b, void *stream) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->warm || stale(b)) {
      const int e = warm_up(b, s);
      if (e) return e;
    }
    if (!b->exec) {
      const int e = capture(b);
      if (e) return e;
    }
    NAPMO_TRY_CUDA(cudaGraphLaunch(b->exec, s), "batch launch");
    return kOk;
  });
}

// Autotuner of the batch's launch shape (see the file comment), timed on the
// densities currently in the batch's D buffers (the cost of a truncated
// Poisson evaluation depends on them).  Returns the chosen nstream, budget
// (CTAs) and the time of one batch build in ms.
int napmo_fock_batch_tune(FockBatch *b, void *stream, int reps, int *nstream_out,
                          int *budget_out, double *ms_out) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    NAPMO_REQUIRE(reps >= 1, "reps must be >= 1");
    int dev = 0, sms = 148;
    NAPMO_TRY_CUDA(cudaGetDevice(&dev), "device");
    NAPMO_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SMs");
    if (!b->warm || stale(b)) {
      const int e = warm_up(b, s);
      if (e) return e;
    }
    bool any_i8 = false;
    for (auto *p : b->plans) any_i8 = any_i8 || fock_plan_int8(p) != nullptr;
    std::vector<int> budgets = {sms};
    if (any_i8) budgets = {sms, sms / 2, sms / 4, sms / 8};
    cudaEvent_t e0, e1;
    NAPMO_TRY_CUDA(cudaEventCreate(&e0), "events");
    NAPMO_TRY_CUDA(cudaEventCreate(&e1), "events");
    float best = -1.0f;
    int best_ns = b->nstream, best_budget = b->budget;
    int st = kOk;
    for (int ns : {1, 2, 4, 8, 16, 32}) {
      if (ns > (int)b->plans.size() && ns > 1) break;
      if (b->mode == 1 && ns > 1) break;  // stage launches: no capture streams to choose
      for (int bud : budgets) {
        b->nstream = ns;
        if ((st = set_budgets(b, bud))) break;
        if (b->mode == 1 && (st = warm_up(b, s))) break;  // stage tables hold the budgets
        if ((st = capture(b))) break;
        cudaGraphLaunch(b->exec, s);
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps; ++r) cudaGraphLaunch(b->exec, s);
        cudaEventRecord(e1, s);
        const cudaError_t ce = cudaEventSynchronize(e1);
        if (ce != cudaSuccess) {
          st = cuda_status(ce, "batch tuning");
          break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= reps;
        if (best < 0.0f || ms < best) {
          best = ms;
          best_ns = ns;
          best_budget = bud;
        }
      }
      if (st) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    b->nstream = best_ns;
    if ((st = set_budgets(b, best_budget))) return st;
    if (b->mode == 1 && (st = warm_up(b, s))) return st;
    if ((st = capture(b))) return st;
    b->tuned_ms = best;
    if (nstream_out) *nstream_out = best_ns;
    if (budget_out) *budget_out = best_budget;
    if (ms_out) *ms_out = best;
    return kOk;
  });
}

// Build mode: 0 = the molecules' own launch chains spread over capture
// streams; 1 = one launch per stage for the whole batch (persistent density
// and quadrature launches over device work queues, one Poisson plan over all
// grids; FP64 plans).  Takes effect at the next build (re-warms and
// recaptures).
int napmo_fock_batch_set_mode(FockBatch *b, int mode) {
  return guarded([&] {
    NAPMO_REQUIRE(mode == 0 || mode == 1, "mode must be 0 (streams) or 1 (stages)");
    b->mode = mode;
    b->warm = false;
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    return kOk;
  });
}

// Mode 1: runs the density stage with a work queue that is never posted, so
// that every CTA's bounded wait runs out after timeout_ns; *status receives
// the queue's error word (5 = a wait ran out).  The batch stays usable.
int napmo_fock_batch_queue_selftest(FockBatch *b, double timeout_s, void *stream,
                                    int *status) {
  return guarded([&] {
    cudaStream_t s = (cudaStream_t)stream;
    NAPMO_REQUIRE(b->mode == 1, "the work queues belong to mode 1");
    NAPMO_REQUIRE(timeout_s > 0.0 && timeout_s <= 10.0, "timeout must be in (0, 10] s");
    if (!b->warm || stale(b)) {
      const int e = warm_up(b, s);
      if (e) return e;
    }
    return stage_batch_queue_selftest(b->stage, (unsigned long long)(timeout_s * 1e9), s, status);
  });
}

// Mode 1: error word of the work queues since the last call (0 or 5); clears it.
int napmo_fock_batch_status(FockBatch *b, void *stream, int *status) {
  return guarded([&] {
    *status = 0;
    if (b->stage) return stage_batch_status(b->stage, (cudaStream_t)stream, status);
    return kOk;
  });
}

// Current launch shape (nstream, budget; budget 0 = kernels' default).
int napmo_fock_batch_config(FockBatch *b, int *nstream, int *budget) {
  *nstream = b->nstream;
  *budget = b->budget;
  return kOk;
}

}  // extern "C"
