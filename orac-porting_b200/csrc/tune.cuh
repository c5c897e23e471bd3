// Shared pieces of the pair-kernel autotuner (tune.cu, batch.cu).
#pragma once
#include <string>
#include <vector>

#include "common.cuh"

struct PairTune {
  int lpg_m, lpg_lh, minb;
};

int tune_candidates(int maxg, std::vector<PairTune>* out);
void tune_apply(orac_gpu_ctx* ctx, const PairTune& t);
std::string tune_signature(const std::vector<orac_gpu_ctx*>& ctxs, const char* what);
bool tune_cache_find(const char* path, const std::string& sig, PairTune* t, double* ms);
void tune_cache_add(const char* path, const std::string& sig, const PairTune& t, double ms);
