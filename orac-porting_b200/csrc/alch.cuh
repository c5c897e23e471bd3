// Lambda tables and charges of the alchemy variant, shared by the host
// setters and the device-side lambda schedule of non-equilibrium runs.
#pragma once
#include <cmath>

#include "common.cuh"

// alch_set (src/force_alchemy_shifted.f:732-790): [0][t+4] soft-core shift,
// [1][t+4] scale, t = ss_i + ss_j of the pair
__host__ __device__ inline void alch_set(double f[2][9], double ladd, double lrm, int intramol, int ljintra, int qq) {
  for (int k = 0; k < 2; k++)
    for (int t = 0; t < 9; t++) f[k][t] = 0.0;
  const double la = fabs(ladd), lr = fabs(lrm);
  auto put = [&](int t, double a, double b) {
    f[0][t + 4] = a;
    f[1][t + 4] = b;
  };
  put(2, 0.0, 1.0);
  put(3, la, 1.0 - la);
  put(-1, lr, 1.0 - lr);
  if (intramol && qq) {
    put(4, la * la, 1.0 - la * la);
    put(-4, lr * lr, 1.0 - lr * lr);
  } else if (intramol && !ljintra) {
    put(4, la, 1.0 - la);
    put(-4, lr, 1.0 - lr);
  } else {
    put(4, 0.0, 1.0);
    put(-4, 0.0, 1.0);
  }
  put(0, 0.0, 0.0);
}

// chrgec of mts_furier_alchemy (src/mts_furier_alchemy.f:96-111)
__host__ __device__ inline double scaled_charge(double q, double lq) {
  const double a = fabs(lq);
  if (a == 1.0) return 0.0;
  if (a == 0.0) return q;
  return (1.0 - a) * q;
}

// FP32 copies of the current tables
__host__ __device__ inline void alch_dyn_f32(AlchDyn* D) {
  for (int k = 0; k < 2; k++)
    for (int t = 0; t < 9; t++) {
      D->af[k][t] = (float)D->f[k][t];
      D->afq[k][t] = (float)D->fq[k][t];
    }
}

// upload ctx->at's lambda tables to the device copy the pair kernel reads
int alch_upload_tables(orac_gpu_ctx* ctx);
