// Autotuner of the real-space kernel's launch configuration: lanes per i
// group on the M shell and on the L/H shells (16 or 32) and resident blocks
// per SM (5, 6 or 8).  A candidate is timed on the real workload -- the
// batch's captured step graphs, or one context's steps -- with CUDA events
// on its stream; the fastest is applied and appended to a cache file keyed
// by the device and the workload's shape, so that the next run with the
// same shape applies it without timing.  The forces do not depend on the
// configuration (fixed-point sums), so tuning changes speed only; the
// trial steps are real MD steps of the systems.
#include <fstream>
#include <sstream>
#include <string>

#include "common.cuh"
#include "tune.cuh"

int tune_candidates(int maxg, std::vector<PairTune>* out) {
  out->clear();
  if (maxg > 4) {  // groups of up to 8 atoms: one build (a warp per group)
    out->push_back({32, 32, 6});
    return ORAC_OK;
  }
  const int lp[2] = {16, 32}, mb[3] = {5, 6, 8};
  for (int m : lp)
    for (int l : lp)
      for (int b : mb) out->push_back({m, l, b});
  return ORAC_OK;
}

void tune_apply(orac_gpu_ctx* ctx, const PairTune& t) {
  if (ctx->tune_lpg_m != t.lpg_m || ctx->tune_lpg_lh != t.lpg_lh || ctx->tune_minb != t.minb) {
    ctx->tune_lpg_m = t.lpg_m;
    ctx->tune_lpg_lh = t.lpg_lh;
    ctx->tune_minb = t.minb;
    ctx->param_gen++;  // the step graphs hold the kernel choice: captured again
  }
}

std::string tune_signature(const std::vector<orac_gpu_ctx*>& ctxs, const char* what) {
  cudaDeviceProp p;
  std::string dev = "gpu";
  if (!ctxs.empty() && cudaGetDeviceProperties(&p, ctxs[0]->device) == cudaSuccess) dev = p.name;
  for (auto& ch : dev)
    if (ch == ' ') ch = '_';
  long long atoms = 0, amax = 0;
  int maxg = 0, var = 0;
  for (auto* c : ctxs) {
    atoms += c->N;
    amax = c->N > amax ? c->N : amax;
    maxg = c->maxg > maxg ? c->maxg : maxg;
    var |= 1 << c->variant;
  }
  std::ostringstream s;
  s << dev << ";" << what << ";systems=" << ctxs.size() << ";atoms=" << atoms << ";max_atoms=" << amax
    << ";maxg=" << maxg << ";variants=" << var;
  return s.str();
}

bool tune_cache_find(const char* path, const std::string& sig, PairTune* t, double* ms) {
  if (!path || !*path) return false;
  std::ifstream f(path);
  std::string line;
  bool found = false;
  while (std::getline(f, line)) {  // the last entry of a signature wins
    std::istringstream in(line);
    std::string s;
    PairTune c;
    double m = 0.0;
    if (in >> s >> c.lpg_m >> c.lpg_lh >> c.minb >> m && s == sig) {
      *t = c;
      if (ms) *ms = m;
      found = true;
    }
  }
  return found;
}

void tune_cache_add(const char* path, const std::string& sig, const PairTune& t, double ms) {
  if (!path || !*path) return;
  std::ofstream f(path, std::ios::app);
  f << sig << " " << t.lpg_m << " " << t.lpg_lh << " " << t.minb << " " << ms << "\n";
}

extern "C" {

int orac_gpu_set_pair_tuning(orac_gpu_ctx* ctx, int lpg_m, int lpg_lh, int minb) {
  if (!ctx) return ORAC_ERR_PARAM;
  auto ok_lpg = [](int v) { return v == 0 || v == 16 || v == 32; };
  if (!ok_lpg(lpg_m) || !ok_lpg(lpg_lh) || !(minb == 0 || minb == 5 || minb == 6 || minb == 8))
    return ctx_fail(ctx, ORAC_ERR_PARAM, "pair tuning lpg_m %d, lpg_lh %d (0, 16, 32), minb %d (0, 5, 6, 8)", lpg_m,
                    lpg_lh, minb);
  tune_apply(ctx, {lpg_m, lpg_lh, minb});
  return ORAC_OK;
}

int orac_gpu_get_pair_tuning(orac_gpu_ctx* ctx, int* out3) {
  if (!ctx || !out3) return ORAC_ERR_PARAM;
  out3[0] = ctx->tune_lpg_m ? ctx->tune_lpg_m : (ctx->shared_device ? 16 : 32);
  out3[1] = ctx->tune_lpg_lh ? ctx->tune_lpg_lh : 32;
  out3[2] = ctx->tune_minb ? ctx->tune_minb : (ctx->shared_device ? 8 : 6);
  return ORAC_OK;
}

// One context alone: every candidate runs `trial` outer steps after the
// same number of warm-up steps (which capture its step graphs).
int orac_gpu_tune(orac_gpu_ctx* ctx, int trial, const char* cache_path, int force, int* out3, double* ms_per_step) {
  if (!ctx || trial < 1) return ORAC_ERR_PARAM;
  CK(cudaSetDevice(ctx->device));
  const std::string sig = tune_signature({ctx}, "alone");
  PairTune best{0, 0, 0};
  double best_ms = 0.0;
  if (!force && tune_cache_find(cache_path, sig, &best, &best_ms)) {
    tune_apply(ctx, best);
  } else {
    std::vector<PairTune> cand;
    tune_candidates(ctx->maxg, &cand);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int rc = ORAC_OK;
    for (const PairTune& c : cand) {
      tune_apply(ctx, c);
      if ((rc = orac_gpu_md_run_async(ctx, trial)) || (rc = orac_gpu_md_collect(ctx))) break;
      if (cudaEventRecord(e0, ctx->stream) != cudaSuccess) rc = ORAC_ERR_CUDA;
      if (!rc && (rc = orac_gpu_md_run_async(ctx, trial))) break;
      if (!rc && cudaEventRecord(e1, ctx->stream) != cudaSuccess) rc = ORAC_ERR_CUDA;
      if (!rc) rc = orac_gpu_md_collect(ctx);
      if (rc) break;
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = ORAC_ERR_CUDA;
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
    tune_apply(ctx, best);
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

}  // extern "C"
