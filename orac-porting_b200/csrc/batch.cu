// Batched execution of many systems: every context keeps its own state,
// lists and step graph; the batch splices those graphs as independent
// child nodes of one parent graph, so one graph launch advances all
// systems by one outer step and the device runs their kernels
// concurrently.  This is the on-device replacement for running ORAC
// replicas (HREM states, alchemical windows) as separate MPI ranks
// (src/rem.f90, src/orac_mpi.f90).
#include "common.cuh"

struct MdState;

// md.cu: captured step graph of a context (kind 0: plain step, 1: step with
// list update); captures it on first use
int md_step_graph(orac_gpu_ctx* ctx, int kind, cudaGraph_t* out);
int md_advance(orac_gpu_ctx* ctx, int nsteps);
long long md_step_index(orac_gpu_ctx* ctx);
int md_nupdte(orac_gpu_ctx* ctx);
int md_check_flags(orac_gpu_ctx* ctx);

struct orac_gpu_batch {
  std::vector<orac_gpu_ctx*> ctx;
  std::vector<unsigned> gen;  // each context's param_gen when the batch was built
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  cudaGraph_t graph[2] = {nullptr, nullptr};
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
  for (int k = 0; k < 2; k++) {
    if (b->exec[k]) cudaGraphExecDestroy(b->exec[k]);
    if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
  }
  if (b->stream) cudaStreamDestroy(b->stream);
  for (auto* c : b->ctx) c->shared_device = false;
  delete b;
  return ORAC_OK;
}

// Advance every system of the batch by nsteps outer steps with one graph
// launch per step.  All systems must have been set up with orac_gpu_md_setup
// and share the list-update period and the current step index.
int orac_gpu_batch_run(orac_gpu_batch* b, int nsteps) {
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
    const int kind = (step % nup == 0 && step > 0) ? 1 : 0;
    if (int rc = build_kind(b, kind)) return rc;
    if (cudaGraphLaunch(b->exec[kind], b->stream) != cudaSuccess) return bfail(b, ORAC_ERR_CUDA, "cudaGraphLaunch");
    for (auto* c : b->ctx) md_advance(c, 1);
  }
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

}  // extern "C"
