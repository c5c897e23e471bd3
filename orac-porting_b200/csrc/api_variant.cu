// Variants of the shell kernel: the REM segment scaling of force_rem
// (src/force_REM.f, seg_select src/rem.f90:631-645) and the soft-core
// alchemy of force_alchemy (src/force_alchemy.f with alch_set,
// src/force_alchemy_shifted.f:732-790), selected as mts_forces does
// (src/mts_forces.f:118-153).
#include <cmath>

#include "alch.cuh"
#include "common.cuh"

namespace {

// derivative of alch_set's tables with respect to a control lambda that
// moves ladd and lrm at rates dla and dlr (d|l|/dl taken as +1 at l = 0)
void alch_set_d(double d[2][9], double ladd, double lrm, double dla, double dlr, int intramol, int ljintra, int qq) {
  for (int k = 0; k < 2; k++)
    for (int t = 0; t < 9; t++) d[k][t] = 0.0;
  const double sa = ladd < 0 ? -1.0 : 1.0, sr = lrm < 0 ? -1.0 : 1.0;
  const double la = std::fabs(ladd), lr = std::fabs(lrm);
  auto put = [&](int t, double a, double b) {
    d[0][t + 4] = a;
    d[1][t + 4] = b;
  };
  put(3, sa * dla, -sa * dla);
  put(-1, sr * dlr, -sr * dlr);
  if (intramol && qq) {
    put(4, 2.0 * la * sa * dla, -2.0 * la * sa * dla);
    put(-4, 2.0 * lr * sr * dlr, -2.0 * lr * sr * dlr);
  } else if (intramol && !ljintra) {
    put(4, sa * dla, -sa * dla);
    put(-4, sr * dlr, -sr * dlr);
  }
}

__global__ void k_variant_out(const double* __restrict__ acc, int variant, int forces_on, double* __restrict__ x) {
  pdl_enter();
  if (threadIdx.x != 0) return;
  for (int k = 0; k < 5; k++) x[k] = 0.0;  // x[5] is the PME's
  if (!forces_on) return;
  if (variant == VAR_REM) x[0] = acc[ACC_X];
  if (variant == VAR_ALCH) {
    double u = 0.0;
    for (int k = 0; k < 6; k++) u += acc[ACC_CONF + k];
    x[1] = u - acc[ACC_X] - acc[ACC_X + 1];
    x[2] = acc[ACC_X];
    x[3] = acc[ACC_X + 1];
    x[4] = acc[ACC_X + 2];
  }
}

int build_vflag(orac_gpu_ctx* ctx) {
  const int N = ctx->N;
  ctx->h_vflag.assign(N, 0);
  for (int a = 0; a < N; a++) {
    unsigned char f = 0;
    if (ctx->h_mass[a] >= ctx->massinfty) f |= VF_MINF;
    if (!ctx->h_rem.empty() && ctx->h_rem[a]) f |= VF_REM;
    const int ss = ctx->h_ssal.empty() ? 1 : ctx->h_ssal[a];
    f |= (unsigned char)((ss + 4) << VF_SSHIFT);
    ctx->h_vflag[a] = f;
  }
  if (!ctx->d_vflag && dev_alloc(ctx, &ctx->d_vflag, N)) return ORAC_ERR_CUDA;
  CK(cudaMemcpy(ctx->d_vflag, ctx->h_vflag.data(), N, cudaMemcpyHostToDevice));
  return ORAC_OK;
}

int upload_alch_charges(orac_gpu_ctx* ctx, const double* dlam) {
  const int N = ctx->N;
  std::vector<double> qc(N), q0(N), dq(N, 0.0);
  double sq = 0.0;
  for (int a = 0; a < N; a++) {
    const int ss = ctx->h_ssal[a];
    // lambdaq of added atoms is laddq, of removed atoms -lrmq (src/mtsmd.f:747,755)
    const double lq = ss == 2 ? ctx->lam[2] : (ss == -2 ? -ctx->lam[3] : 0.0);
    const double lq0 = ss == 2 ? ctx->lam[6] : (ss == -2 ? -ctx->lam[7] : 0.0);
    qc[a] = scaled_charge(ctx->h_charge[a], lq);
    q0[a] = scaled_charge(ctx->h_charge[a], lq0);
    if (dlam) {
      // d/dlambda of (1 - |lambdaq|) q with lambdaq = laddq or -lrmq
      if (ss == 2) dq[a] = -(ctx->lam[2] < 0 ? -1.0 : 1.0) * ctx->h_charge[a] * dlam[2];
      if (ss == -2) dq[a] = -(ctx->lam[3] < 0 ? -1.0 : 1.0) * ctx->h_charge[a] * dlam[3];
    }
    if (ctx->h_ss[a] == 1) sq += 2.0 * qc[a] * dq[a];
  }
  // cself_alchemy (src/cself_alchemy.f): -alpha/sqrt(pi) sum_slt qc^2 (1 - erfc(kcut/2 alpha))
  {
    const double ar = ctx->rkcut / (2.0 * ctx->alphal);
    const double qt = 1.0 / (1.0 + 0.3275911 * ar);
    const double erfcst =
        ((((1.0614054 * qt - 1.453152) * qt + 1.4214137) * qt - 0.28449674) * qt + 0.2548296) * qt * std::exp(-ar * ar);
    ctx->self_dudl = -sq * ctx->alphal / std::sqrt(4.0 * std::atan(1.0)) * (1.0 - erfcst);
  }
  if (!ctx->d_qc && (dev_alloc(ctx, &ctx->d_qc, N) || dev_alloc(ctx, &ctx->d_q0, N))) return ORAC_ERR_CUDA;
  CK(cudaMemcpy(ctx->d_qc, qc.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_q0, q0.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  ctx->q0_differs = qc != q0;
  {
    // per-atom lambdas of fnb14_alchemy / ferrf_alchemy_add and the
    // derivatives of their couplings 1 - |lambda| (added: ladd, removed:
    // -lrm, src/mtsmd.f:746-754)
    std::vector<double4> l4(N);
    const double d0[4] = {0, 0, 0, 0};
    const double* d = dlam ? dlam : d0;
    for (int a = 0; a < N; a++) {
      const int ss = ctx->h_ssal[a];
      const double ll = ss == 2 ? ctx->lam[0] : (ss == -2 ? -ctx->lam[1] : 0.0);
      const double lq = ss == 2 ? ctx->lam[2] : (ss == -2 ? -ctx->lam[3] : 0.0);
      const double sl = ss == 2 ? (ctx->lam[0] < 0 ? -1.0 : 1.0) * d[0] : (ss == -2 ? (ctx->lam[1] < 0 ? -1.0 : 1.0) * d[1] : 0.0);
      const double sq = ss == 2 ? (ctx->lam[2] < 0 ? -1.0 : 1.0) * d[2] : (ss == -2 ? (ctx->lam[3] < 0 ? -1.0 : 1.0) * d[3] : 0.0);
      l4[a] = make_double4(ll, lq, -sl, -sq);
    }
    if (!ctx->d_lam4 && dev_alloc(ctx, &ctx->d_lam4, N)) return ORAC_ERR_CUDA;
    CK(cudaMemcpy(ctx->d_lam4, l4.data(), sizeof(double4) * N, cudaMemcpyHostToDevice));
  }
  if (dlam) {
    if (!ctx->d_dq && dev_alloc(ctx, &ctx->d_dq, N)) return ORAC_ERR_CUDA;
    CK(cudaMemcpy(ctx->d_dq, dq.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  } else if (ctx->d_dq) {
    dev_free(ctx, ctx->d_dq);
    ctx->d_dq = nullptr;
  }
  return ORAC_OK;
}

}  // namespace

int alch_upload_tables(orac_gpu_ctx* ctx) {
  AlchDyn D;
  const AlchTables& T = ctx->at;
  for (int k = 0; k < 2; k++)
    for (int t = 0; t < 9; t++) {
      D.f[k][t] = T.f[k][t];
      D.fq[k][t] = T.fq[k][t];
      D.f0[k][t] = T.f0[k][t];
      D.fq0[k][t] = T.fq0[k][t];
      D.df[k][t] = T.df[k][t];
      D.dfq[k][t] = T.dfq[k][t];
    }
  alch_dyn_f32(&D);
  if (!ctx->d_ad && dev_alloc(ctx, &ctx->d_ad, 1)) return ORAC_ERR_CUDA;
  // stream-ordered: a step graph still running reads the old tables
  CK(cudaMemcpyAsync(ctx->d_ad, &D, sizeof(D), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return ORAC_OK;
}


void variant_fill(const orac_gpu_ctx* ctx, PairArgs* a) {
  a->variant = ctx->variant;
  if (ctx->variant == VAR_STD) return;
  a->vflag = ctx->d_vflag;
  a->rem_kind = ctx->rem_kind;
  a->remf = ctx->d_remf;
  if (ctx->variant == VAR_ALCH) {
    a->soft = ctx->d_soft;
    a->softd = ctx->d_softd;
    a->at = ctx->at;
    a->qsoft = (float)ctx->at.qsoft;
    a->ljsoft = (float)ctx->at.ljsoft;
    a->qshift = (float)ctx->at.qshift;
    a->ljshift_s = (float)ctx->at.ljshift_s;
    a->ad = ctx->d_ad;
  }
}

int variant_out_launch(orac_gpu_ctx* ctx, int forces_on) {
  if (!ctx->d_xtra && dev_alloc(ctx, &ctx->d_xtra, 8)) return ORAC_ERR_CUDA;
  orac_launch(k_variant_out, 1, 32, 0, ctx->stream, ctx->d_acc, ctx->variant, forces_on, ctx->d_xtra);
  CKL();
  return ORAC_OK;
}

// listqq of src/initialize_lambda.f:62-139 from the species and the
// context's pair lists: every pair of alchemical atoms that is no bond,
// constraint, 1-3 or 1-4 pair, facQ 1 within a species, 0 across.  Built
// when the MD driver is set up (the constraints are known then) and again
// when the species change.
int alch_listqq_build(orac_gpu_ctx* ctx) {
  const BondedDev& B = ctx->bd;
  std::vector<int> iat;  // ORAC's order: added atoms, then removed ones
  for (int a = 0; a < ctx->N; a++)
    if (ctx->h_ssal.size() == (size_t)ctx->N && ctx->h_ssal[a] == 2) iat.push_back(a + 1);
  for (int a = 0; a < ctx->N; a++)
    if (ctx->h_ssal.size() == (size_t)ctx->N && ctx->h_ssal[a] == -2) iat.push_back(a + 1);
  std::unordered_map<long long, char> excl;
  auto key = [](int i, int j) { return i < j ? ((long long)i << 32) | (unsigned)j : ((long long)j << 32) | (unsigned)i; };
  const int* lists[4] = {B.pbond, B.pcn, B.p13, B.p14};
  const int n[4] = {B.nb, B.ncn, B.n13, B.n14};
  for (int k = 0; k < 4; k++) {
    if (!lists[k] || n[k] <= 0) continue;
    std::vector<int> h(2 * (size_t)n[k]);
    CK(cudaMemcpy(h.data(), lists[k], sizeof(int) * h.size(), cudaMemcpyDeviceToHost));
    for (int q = 0; q < n[k]; q++) excl[key(h[2 * q], h[2 * q + 1])] = 1;
  }
  std::vector<int> out;
  for (size_t a = 0; a + 1 < iat.size(); a++)
    for (size_t b = a + 1; b < iat.size(); b++) {
      if (excl.count(key(iat[a], iat[b]))) continue;
      out.push_back(iat[a]);
      out.push_back(iat[b]);
      out.push_back(ctx->h_ssal[iat[a] - 1] == ctx->h_ssal[iat[b] - 1] ? 1 : 0);
    }
  ctx->nlistqq = (int)(out.size() / 3);
  if (ctx->nlistqq > 0) {
    if (dev_alloc(ctx, &ctx->d_listqq, out.size())) return ORAC_ERR_CUDA;
    CK(cudaMemcpy(ctx->d_listqq, out.data(), sizeof(int) * out.size(), cudaMemcpyHostToDevice));
  }
  return ORAC_OK;
}

void variant_free(orac_gpu_ctx* ctx) {
  void* p[] = {ctx->d_vflag, ctx->d_soft, ctx->d_softd, ctx->d_qc, ctx->d_q0, ctx->d_xtra, ctx->d_dq,
               ctx->d_lam4, ctx->d_listqq, ctx->d_remf, ctx->d_ad, ctx->d_lam40, ctx->d_ne, ctx->d_ne_alist};
  for (void* q : p)
    if (q) dev_free(ctx, q);
}

extern "C" {

int orac_gpu_set_rem(orac_gpu_ctx* ctx, const int* rematom, int kind, double rem_factor) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  CK(cudaSetDevice(ctx->device));
  if (!rematom) {
    bump.arm();
    if (ctx->variant == VAR_REM) ctx->variant = VAR_STD;
    ctx->h_rem.clear();
    return ORAC_OK;
  }
  if (kind < 0 || kind > 2) return ctx_fail(ctx, ORAC_ERR_PARAM, "REM segment kind %d (0, 1 or 2)", kind);
  if (!(rem_factor >= 0.0)) return ctx_fail(ctx, ORAC_ERR_PARAM, "rem_factor %g", rem_factor);
  bump.arm();
  ctx->h_rem.assign(ctx->N, 0);
  for (int a = 0; a < ctx->N; a++) ctx->h_rem[a] = rematom[a] ? 1 : 0;
  ctx->rem_kind = kind;
  ctx->rem_factor = rem_factor;
  {
    const float f = (float)rem_factor;
    if (!ctx->d_remf && dev_alloc(ctx, &ctx->d_remf, 1)) return ORAC_ERR_CUDA;
    CK(cudaMemcpy(ctx->d_remf, &f, sizeof(float), cudaMemcpyHostToDevice));
  }
  if (int rc = build_vflag(ctx)) return rc;
  ctx->variant = VAR_REM;
  return ORAC_OK;
}

int orac_gpu_set_rem_factor_async(orac_gpu_ctx* ctx, double rem_factor, void* stream) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (ctx->variant != VAR_REM || !ctx->d_remf) return ctx_fail(ctx, ORAC_ERR_STATE, "orac_gpu_set_rem first");
  if (!(rem_factor >= 0.0)) return ctx_fail(ctx, ORAC_ERR_PARAM, "rem_factor %g", rem_factor);
  CK(cudaSetDevice(ctx->device));
  ctx->rem_factor = rem_factor;
  ctx->h_remf = (float)rem_factor;  // staged: the copy reads it when the stream gets there
  CK(cudaMemcpyAsync(ctx->d_remf, &ctx->h_remf, sizeof(float), cudaMemcpyHostToDevice,
                     stream ? (cudaStream_t)stream : ctx->stream));
  return ORAC_OK;
}

int orac_gpu_set_alchemy(orac_gpu_ctx* ctx, const int* ss_alchemy, const double* rmin, const double* epsm,
                         double qsoft, double ljsoft, int opls) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  CK(cudaSetDevice(ctx->device));
  if (!ss_alchemy) {
    bump.arm();
    if (ctx->variant == VAR_ALCH) ctx->variant = VAR_STD;
    ctx->h_ssal.clear();
    return ORAC_OK;
  }
  if (!rmin || !epsm) return ctx_fail(ctx, ORAC_ERR_PARAM, "rmin and epsm are required");
  const int N = ctx->N;
  std::vector<float2> sf(N);
  std::vector<double2> sd(N);
  for (int a = 0; a < N; a++) {
    const int s = ss_alchemy[a];
    if (s != 1 && s != 2 && s != -2)
      return ctx_fail(ctx, ORAC_ERR_PARAM, "ss_alchemy(%d) = %d (1 normal, 2 added, -2 removed)", a + 1, s);
    if (!(rmin[a] >= 0.0) || !(epsm[a] >= 0.0))
      return ctx_fail(ctx, ORAC_ERR_PARAM, "rmin/epsm of atom %d", a + 1);
    sf[a] = make_float2((float)rmin[a], (float)(2.0 * std::sqrt(epsm[a])));
    sd[a] = make_double2(rmin[a], epsm[a]);
  }
  bump.arm();
  ctx->h_ssal.assign(ss_alchemy, ss_alchemy + N);
  ctx->nlistqq = -1;  // the species changed: listqq is built again
  if (!ctx->d_soft && (dev_alloc(ctx, &ctx->d_soft, N) || dev_alloc(ctx, &ctx->d_softd, N))) return ORAC_ERR_CUDA;
  CK(cudaMemcpy(ctx->d_soft, sf.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_softd, sd.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
  ctx->at.qsoft = qsoft;
  ctx->at.ljsoft = ljsoft;
  ctx->at.opls = opls ? 1 : 0;
  if (int rc = build_vflag(ctx)) return rc;
  ctx->variant = VAR_ALCH;
  const double zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  return orac_gpu_set_lambda(ctx, zero, 0, 0, nullptr);
}

int orac_gpu_set_alchemy_shift(orac_gpu_ctx* ctx, int shifted, double qshift, double ljshift) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx) return ORAC_ERR_PARAM;
  if (shifted && !(qshift >= 0.0 && ljshift >= 0.0))
    return ctx_fail(ctx, ORAC_ERR_PARAM, "qshift %g and ljshift %g must be >= 0", qshift, ljshift);
  bump.arm();
  ctx->at.shifted = shifted ? 1 : 0;
  ctx->at.qshift = shifted ? qshift : 0.0;
  // ORAC's two6 = 2.d0**(1./6.), the exponent a single-precision constant
  ctx->at.ljshift_s = shifted ? ljshift * std::pow(2.0, (double)(1.0f / 6.0f)) : 0.0;
  return ORAC_OK;
}

int orac_gpu_set_lambda(orac_gpu_ctx* ctx, const double* lam, int intramol, int ljintra, const double* dlam) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx) return ORAC_ERR_PARAM;
  if (ctx->h_ssal.empty()) return ctx_fail(ctx, ORAC_ERR_STATE, "orac_gpu_set_alchemy first");
  if (!lam) return ctx_fail(ctx, ORAC_ERR_PARAM, "lam is required");
  for (int k = 0; k < 8; k++)
    if (!(std::fabs(lam[k]) <= 1.0)) return ctx_fail(ctx, ORAC_ERR_PARAM, "lambda %d = %g outside [-1, 1]", k, lam[k]);
  CK(cudaSetDevice(ctx->device));
  bump.arm();
  for (int k = 0; k < 8; k++) ctx->lam[k] = lam[k];
  ctx->alch_intramol = intramol ? 1 : 0;
  const double d0[4] = {0, 0, 0, 0};
  const double* d = dlam ? dlam : d0;
  AlchTables& T = ctx->at;
  alch_set(T.f, lam[0], lam[1], intramol, ljintra, 0);
  alch_set(T.fq, lam[2], lam[3], intramol, ljintra, 1);
  alch_set(T.f0, lam[4], lam[5], intramol, ljintra, 0);
  alch_set(T.fq0, lam[6], lam[7], intramol, ljintra, 1);
  alch_set_d(T.df, lam[0], lam[1], d[0], d[1], intramol, ljintra, 0);
  alch_set_d(T.dfq, lam[2], lam[3], d[2], d[3], intramol, ljintra, 1);
  if (int rc = alch_upload_tables(ctx)) return rc;
  return upload_alch_charges(ctx, dlam);
}

int orac_gpu_variant_energies(orac_gpu_ctx* ctx, double* out) {
  if (!ctx || !out) return ORAC_ERR_PARAM;
  CK(cudaSetDevice(ctx->device));
  double x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (ctx->d_xtra) {
    CK(cudaMemcpyAsync(x, ctx->d_xtra, sizeof(double) * 6, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  for (int k = 0; k < 5; k++) out[k] = x[k];
  out[5] = ctx->pme_dwrk;
  out[6] = x[5];  // PME dU/dlambda of the last fft_pme
  out[7] = ctx->self_dudl;
  return ORAC_OK;
}

}  // extern "C"
