// Batched execution of many systems: every context keeps its own state,
// lists and step graph; the batch splices those graphs as independent
// child nodes of one parent graph, so one graph launch advances all
// systems by one outer step and the device runs their kernels
// concurrently.  This is the on-device replacement for running ORAC
// replicas (HREM states, alchemical windows) as separate MPI ranks
// (src/rem.f90, src/orac_mpi.f90).
#include "common.cuh"
#include "tune.cuh"

#include <cmath>

struct MdState;

// md.cu: captured step graph of a context (kind bit 0: the step updates the
// lists, bit 1: it writes an energy record); captures it on first use
int md_step_graph(orac_gpu_ctx* ctx, int kind, cudaGraph_t* out);
int md_advance(orac_gpu_ctx* ctx, int nsteps, int kind);
long long md_step_index(orac_gpu_ctx* ctx);
int md_nupdte(orac_gpu_ctx* ctx);
int md_check_flags(orac_gpu_ctx* ctx);

struct orac_gpu_batch {
  std::vector<orac_gpu_ctx*> ctx;
  std::vector<unsigned> gen;  // each context's param_gen when the batch was built
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraph_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
  char err[512] = {0};
  int device = 0;
};

static int bfail(orac_gpu_batch* b, int code, const char* msg) {
  if (b) snprintf(b->err, sizeof(b->err), "%s", msg);
  return code;
}

// parent graph of one step kind: every context's step graph as an
// independent child node
static int build_kind(orac_gpu_batch* b, int kind) {
  if (b->exec[kind]) return ORAC_OK;
  cudaGraph_t parent;
  if (cudaGraphCreate(&parent, 0) != cudaSuccess) return bfail(b, ORAC_ERR_CUDA, "cudaGraphCreate");
  for (auto* c : b->ctx) {
    cudaGraph_t child = nullptr;
    if (int rc = md_step_graph(c, kind, &child)) {
      cudaGraphDestroy(parent);
      return bfail(b, rc, orac_gpu_last_error(c));
    }
    cudaGraphNode_t node;
    if (cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child) != cudaSuccess) {
      cudaGraphDestroy(parent);
      return bfail(b, ORAC_ERR_CUDA, "cudaGraphAddChildGraphNode");
    }
  }
  if (cudaGraphInstantiate(&b->exec[kind], parent, 0) != cudaSuccess) {
    cudaGraphDestroy(parent);
    return bfail(b, ORAC_ERR_CUDA, "cudaGraphInstantiate");
  }
  b->graph[kind] = parent;
  // the systems' own streams must not run work concurrently with the batch
  for (auto* c : b->ctx) cudaStreamSynchronize(c->stream);
  return ORAC_OK;
}

extern "C" {

int orac_gpu_batch_create(orac_gpu_ctx** ctxs, int n, orac_gpu_batch** out) {
  if (!ctxs || n <= 0 || !out) return ORAC_ERR_PARAM;
  orac_gpu_batch* b = new orac_gpu_batch();
  b->device = ctxs[0]->device;
  for (int k = 0; k < n; k++) {
    if (!ctxs[k] || ctxs[k]->device != b->device) {
      delete b;
      return ORAC_ERR_PARAM;
    }
    b->ctx.push_back(ctxs[k]);
    b->gen.push_back(ctxs[k]->param_gen);
  }
  if (cudaSetDevice(b->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return ORAC_ERR_CUDA;
  }
  *out = b;
  // many systems share the device: their pair kernels take the
  // higher-occupancy build (the step graphs are captured again for it)
  for (auto* c : b->ctx) c->shared_device = n > 1;
  // instantiate both step kinds now when every system is set up, so that no
  // step of a run pays for it
  bool ready = true;
  for (auto* c : b->ctx) ready = ready && md_nupdte(c) > 0;
  if (ready)
    for (int kind = 0; kind < 2; kind++)
      if (int rc = build_kind(b, kind)) return rc;
  return ORAC_OK;
}

const char* orac_gpu_batch_last_error(const orac_gpu_batch* b) { return b ? b->err : "null batch"; }

int orac_gpu_batch_destroy(orac_gpu_batch* b) {
  if (!b) return ORAC_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (int k = 0; k < 4; k++) {
    if (b->exec[k]) cudaGraphExecDestroy(b->exec[k]);
    if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
  }
  if (b->stream) cudaStreamDestroy(b->stream);
  for (auto* c : b->ctx) c->shared_device = false;
  delete b;
  return ORAC_OK;
}

// Advance every system of the batch by nsteps outer steps with one graph
// launch per step; with energy_every > 0 every energy_every-th step also
// writes each system's energy record (orac_gpu_md_records).  All systems
// must have been set up with orac_gpu_md_setup and share the list-update
// period and the current step index.
static int batch_run(orac_gpu_batch* b, int nsteps, int energy_every) {
  if (!b) return ORAC_ERR_PARAM;
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, ORAC_ERR_CUDA, "cudaSetDevice");
  const int nup = md_nupdte(b->ctx[0]);
  const long long st0 = md_step_index(b->ctx[0]);
  for (auto* c : b->ctx)
    if (md_nupdte(c) != nup || md_step_index(c) != st0 || nup <= 0)
      return bfail(b, ORAC_ERR_STATE, "batched systems need md_setup, one list-update period and one step index");
  for (size_t k = 0; k < b->ctx.size(); k++)
    if (b->ctx[k]->param_gen != b->gen[k])
      return bfail(b, ORAC_ERR_STATE, "a system's parameters changed after the batch was built: build it again");
  for (int s = 0; s < nsteps; s++) {
    const long long step = md_step_index(b->ctx[0]);
    int kind = (step % nup == 0 && step > 0) ? 1 : 0;
    if (energy_every > 0 && (s + 1) % energy_every == 0) kind |= 2;
    if (int rc = build_kind(b, kind)) return rc;
    if (cudaGraphLaunch(b->exec[kind], b->stream) != cudaSuccess) return bfail(b, ORAC_ERR_CUDA, "cudaGraphLaunch");
    for (auto* c : b->ctx) md_advance(c, 1, kind);
  }
  return ORAC_OK;
}

int orac_gpu_batch_run(orac_gpu_batch* b, int nsteps) { return batch_run(b, nsteps, 0); }

int orac_gpu_batch_run_energy(orac_gpu_batch* b, int nsteps, int energy_every) {
  if (energy_every < 0) return bfail(b, ORAC_ERR_PARAM, "energy_every < 0");
  return batch_run(b, nsteps, energy_every);
}

// Drop the parent graphs and take the members' parameter generations.
// With `eager` the plain and list-update kinds are built again at once from
// the members' current step graphs, so that no step of a later run pays for
// a capture; otherwise each kind is built on its first use.
static int batch_reset_graphs(orac_gpu_batch* b, bool eager) {
  cudaStreamSynchronize(b->stream);
  for (int k = 0; k < 4; k++) {
    if (b->exec[k]) cudaGraphExecDestroy(b->exec[k]);
    if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
    b->exec[k] = nullptr;
    b->graph[k] = nullptr;
  }
  for (size_t k = 0; k < b->ctx.size(); k++) b->gen[k] = b->ctx[k]->param_gen;
  if (eager)
    for (int kind = 0; kind < 2; kind++)
      if (int rc = build_kind(b, kind)) return rc;
  return ORAC_OK;
}

// The autotuner on the batch: every candidate configuration (the same for
// all members) runs `trial` batched steps after `trial` warm-up steps that
// capture its graphs, timed with CUDA events on the batch's stream.
int orac_gpu_batch_tune(orac_gpu_batch* b, int trial, const char* cache_path, int force, int* out3,
                        double* ms_per_step) {
  if (!b || trial < 1) return ORAC_ERR_PARAM;
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, ORAC_ERR_CUDA, "cudaSetDevice");
  const std::string sig = tune_signature(b->ctx, "batch");
  PairTune best{0, 0, 0};
  double best_ms = 0.0;
  if (!force && tune_cache_find(cache_path, sig, &best, &best_ms)) {
    for (auto* c : b->ctx) tune_apply(c, best);
    if (int rc = batch_reset_graphs(b, true)) return rc;
  } else {
    int maxg = 0;
    for (auto* c : b->ctx) maxg = c->maxg > maxg ? c->maxg : maxg;
    std::vector<PairTune> cand;
    tune_candidates(maxg, &cand);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
      return bfail(b, ORAC_ERR_CUDA, "cudaEventCreate");
    int rc = ORAC_OK;
    for (const PairTune& c : cand) {
      for (auto* x : b->ctx) tune_apply(x, c);
      if ((rc = batch_reset_graphs(b, false))) break;
      if ((rc = batch_run(b, trial, 0)) || (rc = orac_gpu_batch_sync(b))) break;
      cudaEventRecord(e0, b->stream);
      if ((rc = batch_run(b, trial, 0))) break;
      cudaEventRecord(e1, b->stream);
      if ((rc = orac_gpu_batch_sync(b))) break;
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = bfail(b, ORAC_ERR_CUDA, "cudaEventElapsedTime");
        break;
      }
      const double per = ms / trial;
      if (best.lpg_m == 0 || per < best_ms) {
        best = c;
        best_ms = per;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    for (auto* c : b->ctx) tune_apply(c, best);
    if (int rc2 = batch_reset_graphs(b, true)) return rc2;
    tune_cache_add(cache_path, sig, best, best_ms);
  }
  if (out3) {
    out3[0] = best.lpg_m;
    out3[1] = best.lpg_lh;
    out3[2] = best.minb;
  }
  if (ms_per_step) *ms_per_step = best_ms;
  return ORAC_OK;
}

// Wait for the batch and check every system's status flags.
int orac_gpu_batch_sync(orac_gpu_batch* b) {
  if (!b) return ORAC_ERR_PARAM;
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bfail(b, ORAC_ERR_CUDA, "batch stream");
  for (auto* c : b->ctx)
    if (int rc = md_check_flags(c)) return bfail(b, rc, orac_gpu_last_error(c));
  return ORAC_OK;
}

void* orac_gpu_batch_stream(orac_gpu_batch* b) { return b ? (void*)b->stream : nullptr; }

// The rem_factor(3) of every member on the batch's stream (ordered with its
// step graphs): what a replica exchange changes.
int orac_gpu_batch_set_rem_factors(orac_gpu_batch* b, const double* factors) {
  if (!b || !factors) return ORAC_ERR_PARAM;
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, ORAC_ERR_CUDA, "cudaSetDevice");
  for (size_t k = 0; k < b->ctx.size(); k++)
    if (int rc = orac_gpu_set_rem_factor_async(b->ctx[k], factors[k], b->stream))
      return bfail(b, rc, orac_gpu_last_error(b->ctx[k]));
  return ORAC_OK;
}

// ORAC's replica-exchange decision (rem_exchange, src/rem.f90:371-537) for
// n replicas and n ensembles of the scaling ladder.  On exchange step
// step_rem the pairs of ensembles (p, p + 1) whose 1-based lower index plus
// step_rem is odd attempt a swap; with pot the replicas' segment energies
// and kT in the same units, delta = (ladder[p+1] - ladder[p]) (pot of the
// replica at p + 1 - pot of the replica at p) / kT, accepted when delta >= 0
// or random <= exp(delta) -- one random number for every pair, as ORAC's
// root broadcasts one.  An accepted pair trades ensembles.
int orac_gpu_rem_exchange(int n, const double* ladder, int* ens, const double* pot, double kT, long long step_rem,
                          double random, int* accepted) {
  if (n < 1 || !ladder || !ens || !pot || !(kT > 0.0)) return ORAC_ERR_PARAM;
  std::vector<int> rep_of(n, -1);
  for (int r = 0; r < n; r++) {
    if (ens[r] < 0 || ens[r] >= n || rep_of[ens[r]] >= 0) return ORAC_ERR_PARAM;  // not a permutation
    rep_of[ens[r]] = r;
  }
  for (int p = 0; p + 1 < n; p++) {
    if (accepted) accepted[p] = 0;
    if (((step_rem + p + 1) & 1LL) == 0) continue;  // ensemble p + 1 (1-based p) is no lower partner now
    const int lo = rep_of[p], hi = rep_of[p + 1];
    const double delta = (ladder[p + 1] - ladder[p]) * (pot[hi] - pot[lo]) / kT;
    if (delta >= 0.0 || random <= std::exp(delta)) {
      ens[lo] = p + 1;
      ens[hi] = p;
      rep_of[p] = hi;
      rep_of[p + 1] = lo;
      if (accepted) accepted[p] = 1;
    }
  }
  return ORAC_OK;
}

}  // extern "C"
