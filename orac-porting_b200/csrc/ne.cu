// Non-equilibrium alchemical runs (ORAC's steered alchemy, test3/test4):
// the lambdas follow a piecewise-linear schedule in time (alchemic,
// src/alchemic.f), updated on the device before every M shell
// (src/mtsmd.f:2963-2999), and the work of each M step is ORAC's sum
// (src/mtsmd.f:3042-3044) of the latest U(lambda) - U(lambda0) of every
// term: the M, L and H shells (force_alchemy's dwrk), the reciprocal level
// (mts_furier_alchemy's dwrk: SPME, erf corrections and self term of the
// scaled charges), ferrf_alchemy_add over listqq and fnb14_alchemy.  The
// lambda state lives in device memory, so the captured step graphs run a
// whole schedule without host round trips, and a batch of contexts runs a
// swarm of such trajectories in one graph launch per step.
#include <cmath>
#include <vector>

#include "alch.cuh"
#include "common.cuh"

namespace {

// alchemic (src/alchemic.f): the slice [trec(i), trec(i+1)] that holds
// rtime (the last one that does), the lambdas linear in time across it;
// before the first point ladd = laddq = 1 and lrm = lrmq = 0, after the last
// point its values.  g = ladd lrm laddq lrmq.
__host__ __device__ void ne_alchemic(const NeDev& ne, double rtime, double* g) {
  g[0] = 1.0;
  g[1] = 0.0;
  g[2] = 1.0;
  g[3] = 0.0;
  int i0 = -1;
  for (int i = 0; i + 1 < ne.ntimes; i++)
    if (rtime >= ne.trec[i] && rtime <= ne.trec[i + 1]) i0 = i;
  if (i0 >= 0) {
    const double ts = ne.trec[i0 + 1] - ne.trec[i0];
    const double dt = rtime - ne.trec[i0];
    // sch rows: ladded laddedq lremoved lremovedq
    g[0] = ne.sch[0][i0] + (ne.sch[0][i0 + 1] - ne.sch[0][i0]) / ts * dt;
    g[1] = ne.sch[2][i0] + (ne.sch[2][i0 + 1] - ne.sch[2][i0]) / ts * dt;
    g[2] = ne.sch[1][i0] + (ne.sch[1][i0 + 1] - ne.sch[1][i0]) / ts * dt;
    g[3] = ne.sch[3][i0] + (ne.sch[3][i0 + 1] - ne.sch[3][i0]) / ts * dt;
  }
  if (rtime > ne.trec[ne.ntimes - 1]) {
    const int n = ne.ntimes - 1;
    g[0] = ne.sch[0][n];
    g[1] = ne.sch[2][n];
    g[2] = ne.sch[1][n];
    g[3] = ne.sch[3][n];
  }
}

// force_alchemy's tables of the current and previous lambdas (alch_set with
// ladd lrm / laddq lrmq and ladd0 ... lrmq0); no control-lambda derivative
__host__ __device__ void ne_tables(const NeDev& ne, AlchDyn* D) {
  alch_set(D->f, ne.g[0], ne.g[1], ne.intramol, ne.ljintra, 0);
  alch_set(D->fq, ne.g[2], ne.g[3], ne.intramol, ne.ljintra, 1);
  alch_set(D->f0, ne.g0[0], ne.g0[1], ne.intramol, ne.ljintra, 0);
  alch_set(D->fq0, ne.g0[2], ne.g0[3], ne.intramol, ne.ljintra, 1);
  for (int k = 0; k < 2; k++)
    for (int t = 0; t < 9; t++) D->df[k][t] = D->dfq[k][t] = 0.0;
  alch_dyn_f32(D);
}

// One block.  Thread 0 advances rtime by the N0 steps of one M step,
// moves the lambdas (the previous ones become lambda0; the added atoms'
// own lambdas move only while ladd or laddq differ from 1, the removed
// atoms' while lrm or lrmq differ from 0, src/mtsmd.f:2974-2998) and
// rebuilds the tables; every thread then sets the PME charges
// (chrgec, chrge0), the per-atom lambdas of the alchemical atoms and the
// solute self term's work (cself_alchemy).
__global__ void k_ne_lambda(NeDev* __restrict__ ne, AlchDyn* __restrict__ ad, int nal, const int4* __restrict__ alist,
                            const double* __restrict__ q, double* __restrict__ qc, double* __restrict__ q0,
                            double* __restrict__ dqc, double4* __restrict__ lam4, double4* __restrict__ lam40,
                            int n0steps) {
  pdl_enter();
  __shared__ double cls[2][4];
  __shared__ double red[32];
  if (threadIdx.x == 0) {
    NeDev& e = *ne;
    e.ninn0 += n0steps;
    e.rtime = e.t0 + (double)e.ninn0 * e.tn0;  // oldtime + ninn0 tn0 (src/mtsmd.f:2751)
    for (int k = 0; k < 4; k++) e.g0[k] = e.g[k];
    ne_alchemic(e, e.rtime, e.g);
    if (e.g[0] != 1.0 || e.g[2] != 1.0) {
      e.pa[2] = e.pa[0];
      e.pa[3] = e.pa[1];
      e.pa[0] = e.g[0];
      e.pa[1] = e.g[2];
    }
    if (e.g[1] != 0.0 || e.g[3] != 0.0) {
      e.pr[2] = e.pr[0];
      e.pr[0] = -e.g[1];
      e.pr[3] = e.pr[1];
      e.pr[1] = -e.g[3];
    }
    ne_tables(e, ad);
    e.dwn[0] = 0.0;
    e.dwn[6] = 0.0;
    for (int k = 0; k < 4; k++) {
      cls[0][k] = e.pa[k];
      cls[1][k] = e.pr[k];
    }
  }
  __syncthreads();
  double s = 0.0;
  for (int i = threadIdx.x; i < nal; i += blockDim.x) {
    const int4 a = alist[i];  // atom, species (+1 added, -1 removed), ss_index
    const double* c = a.y > 0 ? cls[0] : cls[1];
    const double qa = q[a.x];
    const double c1 = scaled_charge(qa, c[1]), c0 = scaled_charge(qa, c[3]);
    qc[a.x] = c1;
    q0[a.x] = c0;
    dqc[a.x] = c1 - c0;
    lam4[a.x] = make_double4(c[0], c[1], 0.0, 0.0);
    lam40[a.x] = make_double4(c[2], c[3], 0.0, 0.0);
    if (a.z == 1) s += c1 * c1 - c0 * c0;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    ne->dself = -ne->selfc * t;
  }
}

// The work of one M step (src/mtsmd.f:3042-3044): the M shell, listqq and
// 1-4 terms of this step, the held L, H and reciprocal terms of their last
// evaluations; then the terms evaluated at this step (bit k of `commit`)
// replace the held ones.  A record (rtime, work) per M step.
__global__ void k_ne_sum(NeDev* __restrict__ ne, int commit) {
  pdl_enter();
  if (threadIdx.x != 0) return;
  NeDev& e = *ne;
  e.wrk += e.dwn[0] + e.dw[1] + e.dw[2] + e.dw[3] + e.dw[4] + e.dw[5] + e.dwn[6] + e.dwn[7];
  for (int k = 0; k < 8; k++)
    if ((commit >> k) & 1) e.dw[k] = e.dwn[k];
  const long long r = e.nrec % NE_REC_CAP;
  e.rec[r][0] = e.rtime;
  e.rec[r][1] = e.wrk;
  e.nrec++;
}

// mts_furier_alchemy's dwrk at one reciprocal evaluation
// (src/mts_furier_alchemy.f:112-186): the SPME energy of chrgec minus that
// of chrge0, summed directly as 2 Re(S conj T) - |T|^2 over the transformed
// grids S of chrgec and T of chrgec - chrge0 (ed[0] holds twice it; the
// difference of two FP32 energies would lose it to rounding), the erf
// corrections of both charge sets (16 slots each) and the self term; into
// the pending slot (the M step's work sum commits it).
__global__ void k_ne_recip(NeDev* __restrict__ ne, const double* __restrict__ ed, const double* __restrict__ fq,
                           const double* __restrict__ f0, int slot) {
  pdl_enter();
  if (threadIdx.x != 0) return;
  double d = 0.5 * ed[0];
  for (int k = 0; k < 16; k++) d += fq[k] - f0[k];
  ne->dwn[slot] = d + ne->dself;
}

}  // namespace

int ne_lambda_launch(orac_gpu_ctx* ctx, int n0steps) {
  orac_launch(k_ne_lambda, 1, 256, 0, ctx->stream, ctx->d_ne, ctx->d_ad, ctx->ne_nal, ctx->d_ne_alist, ctx->d_aqd,
              ctx->d_qc, ctx->d_q0, ctx->d_ne_dq, ctx->d_lam4, ctx->d_lam40, n0steps);
  CKL();
  return ORAC_OK;
}

int ne_sum_launch(orac_gpu_ctx* ctx, int commit) {
  orac_launch(k_ne_sum, 1, 32, 0, ctx->stream, ctx->d_ne, commit);
  CKL();
  return ORAC_OK;
}

int ne_recip_launch(orac_gpu_ctx* ctx, const double* ed, const double* fq, const double* f0, int slot) {
  orac_launch(k_ne_recip, 1, 32, 0, ctx->stream, ctx->d_ne, ed, fq, f0, slot);
  CKL();
  return ORAC_OK;
}

// The run's starting state at t0, set as ORAC sets it when it restarts a
// steered alchemical run (src/mtsmd.f:722-758): the lambdas and their
// previous values are the schedule's at t0; a species whose schedule values
// there are 0 keeps its initial lambdas (added atoms 1, removed atoms 0,
// src/initialize_lambda.f:41-58).  The work and its terms start at 0.
int ne_init(orac_gpu_ctx* ctx, double tn0) {
  NeHost& H = ctx->ne;
  const int N = ctx->N;
  std::vector<NeDev> hv(1);
  NeDev& e = hv[0];
  memset(&e, 0, sizeof(NeDev));
  e.ntimes = (int)H.trec.size();
  for (int i = 0; i < e.ntimes; i++) {
    e.trec[i] = H.trec[i];
    for (int r = 0; r < 4; r++) e.sch[r][i] = H.sch[r][i];
  }
  e.t0 = H.t0;
  e.tn0 = tn0;
  e.rtime = H.t0;
  e.intramol = ctx->alch_intramol;
  e.ljintra = H.ljintra;
  {
    const double ar = ctx->rkcut / (2.0 * ctx->alphal);
    const double qt = 1.0 / (1.0 + 0.3275911 * ar);
    const double erfcst =
        ((((1.0614054 * qt - 1.453152) * qt + 1.4214137) * qt - 0.28449674) * qt + 0.2548296) * qt * std::exp(-ar * ar);
    e.selfc = ctx->alphal / std::sqrt(4.0 * std::atan(1.0)) * (1.0 - erfcst);
  }
  ne_alchemic(e, H.t0, e.g);
  for (int k = 0; k < 4; k++) e.g0[k] = e.g[k];
  const bool add = e.g[0] != 0.0 || e.g[2] != 0.0;
  const bool rm = e.g[1] != 0.0 || e.g[3] != 0.0;
  e.pa[0] = e.pa[2] = add ? e.g[0] : 1.0;
  e.pa[1] = e.pa[3] = add ? e.g[2] : 1.0;
  e.pr[0] = e.pr[2] = rm ? -e.g[1] : 0.0;
  e.pr[1] = e.pr[3] = rm ? -e.g[3] : 0.0;
  // the same lambdas through the host setters: tables, PME charges, lam4
  ctx->lam[0] = e.g[0];
  ctx->lam[1] = e.g[1];
  ctx->lam[2] = e.g[2];
  ctx->lam[3] = e.g[3];
  for (int k = 0; k < 4; k++) ctx->lam[4 + k] = e.g0[k];
  {
    AlchDyn D;
    ne_tables(e, &D);
    for (int k = 0; k < 2; k++)
      for (int t = 0; t < 9; t++) {
        ctx->at.f[k][t] = D.f[k][t];
        ctx->at.fq[k][t] = D.fq[k][t];
        ctx->at.f0[k][t] = D.f0[k][t];
        ctx->at.fq0[k][t] = D.fq0[k][t];
        ctx->at.df[k][t] = ctx->at.dfq[k][t] = 0.0;
      }
  }
  if (int rc = alch_upload_tables(ctx)) return rc;
  std::vector<double> qc(N), q0(N);
  std::vector<double4> l4(N, make_double4(0, 0, 0, 0)), l40(N, make_double4(0, 0, 0, 0));
  std::vector<int4> al;
  for (int a = 0; a < N; a++) {
    const int s = ctx->h_ssal[a];
    const double* c = s == 2 ? e.pa : (s == -2 ? e.pr : nullptr);
    if (!c) {
      qc[a] = q0[a] = ctx->h_charge[a];
      continue;
    }
    qc[a] = scaled_charge(ctx->h_charge[a], c[1]);
    q0[a] = scaled_charge(ctx->h_charge[a], c[3]);
    l4[a] = make_double4(c[0], c[1], 0.0, 0.0);
    l40[a] = make_double4(c[2], c[3], 0.0, 0.0);
    al.push_back(make_int4(a, s > 0 ? 1 : -1, ctx->h_ss[a], 0));
  }
  if (!ctx->d_qc && (dev_alloc(ctx, &ctx->d_qc, N) || dev_alloc(ctx, &ctx->d_q0, N))) return ORAC_ERR_CUDA;
  if (!ctx->d_lam4 && dev_alloc(ctx, &ctx->d_lam4, N)) return ORAC_ERR_CUDA;
  if (!ctx->d_lam40 && dev_alloc(ctx, &ctx->d_lam40, N)) return ORAC_ERR_CUDA;
  if (!ctx->d_ne && dev_alloc(ctx, &ctx->d_ne, 1)) return ORAC_ERR_CUDA;
  if (!ctx->d_ne_dq && dev_alloc(ctx, &ctx->d_ne_dq, N)) return ORAC_ERR_CUDA;
  {
    const PmePlan& P = ctx->pme;
    if (P.qfix && !P.cgsave && dev_alloc(ctx, &ctx->pme.cgsave, (size_t)P.h1 * P.n2 * P.n3)) return ORAC_ERR_CUDA;
  }
  if (dev_alloc(ctx, &ctx->d_ne_alist, al.size())) return ORAC_ERR_CUDA;
  ctx->ne_nal = (int)al.size();
  if (ctx->d_dq) {  // no control-lambda derivative along a schedule
    dev_free(ctx, ctx->d_dq);
    ctx->d_dq = nullptr;
  }
  ctx->q0_differs = qc != q0;
  CK(cudaMemcpy(ctx->d_qc, qc.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_q0, q0.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  {
    std::vector<double> dq(N);
    for (int a = 0; a < N; a++) dq[a] = qc[a] - q0[a];
    CK(cudaMemcpy(ctx->d_ne_dq, dq.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(ctx->d_lam4, l4.data(), sizeof(double4) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_lam40, l40.data(), sizeof(double4) * N, cudaMemcpyHostToDevice));
  if (!al.empty()) CK(cudaMemcpy(ctx->d_ne_alist, al.data(), sizeof(int4) * al.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_ne, &e, sizeof(NeDev), cudaMemcpyHostToDevice));
  return ORAC_OK;
}

extern "C" {

int orac_gpu_md_set_schedule(orac_gpu_ctx* ctx, int ntimes, const double* times, const double* ladded,
                             const double* laddedq, const double* lremoved, const double* lremovedq, double t0,
                             int ljintra) {
  ParamGenBump bump(ctx);  // the step graphs gain the schedule's launches
  if (!ctx) return ORAC_ERR_PARAM;
  if (ctx->variant != VAR_ALCH || ctx->h_ssal.empty())
    return ctx_fail(ctx, ORAC_ERR_STATE, "orac_gpu_set_alchemy first");
  if (md_nupdte(ctx) > 0) return ctx_fail(ctx, ORAC_ERR_STATE, "set the schedule before orac_gpu_md_setup");
  if (ntimes == 0) {
    ctx->ne.on = false;
    bump.arm();
    return ORAC_OK;
  }
  if (ntimes < 2 || ntimes > NE_MAXT || !times || !ladded || !laddedq || !lremoved || !lremovedq)
    return ctx_fail(ctx, ORAC_ERR_PARAM, "schedule of %d points (2..%d, all five arrays)", ntimes, NE_MAXT);
  for (int i = 0; i < ntimes; i++) {
    if (i > 0 && !(times[i] > times[i - 1])) return ctx_fail(ctx, ORAC_ERR_PARAM, "schedule times must increase");
    const double v[4] = {ladded[i], laddedq[i], lremoved[i], lremovedq[i]};
    for (double x : v)
      if (!(std::fabs(x) <= 1.0)) return ctx_fail(ctx, ORAC_ERR_PARAM, "schedule lambda %g outside [-1, 1]", x);
  }
  if (!std::isfinite(t0)) return ctx_fail(ctx, ORAC_ERR_PARAM, "t0");
  bump.arm();
  NeHost& H = ctx->ne;
  H.on = true;
  H.trec.assign(times, times + ntimes);
  const double* s[4] = {ladded, laddedq, lremoved, lremovedq};
  for (int r = 0; r < 4; r++) H.sch[r].assign(s[r], s[r] + ntimes);
  H.t0 = t0;
  H.ljintra = ljintra ? 1 : 0;
  return ORAC_OK;
}

int orac_gpu_md_work(orac_gpu_ctx* ctx, double* out) {
  if (!ctx || !out) return ORAC_ERR_PARAM;
  if (!ctx->d_ne) return ctx_fail(ctx, ORAC_ERR_STATE, "no schedule (orac_gpu_md_set_schedule, then md_setup)");
  CK(cudaSetDevice(ctx->device));
  NeDev* h = new NeDev;
  cudaError_t ce = cudaMemcpyAsync(h, ctx->d_ne, offsetof(NeDev, rec), cudaMemcpyDeviceToHost, ctx->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
  if (ce != cudaSuccess) {
    delete h;
    return ctx_fail(ctx, ORAC_ERR_CUDA, "reading the work: %s", cudaGetErrorString(ce));
  }
  out[0] = h->wrk;
  out[1] = h->rtime;
  for (int k = 0; k < 4; k++) out[2 + k] = h->g[k];
  for (int k = 0; k < 8; k++) out[6 + k] = h->dw[k];
  delete h;
  return ORAC_OK;
}

int orac_gpu_md_work_trace(orac_gpu_ctx* ctx, int max, double* out, int64_t* n_total) {
  if (!ctx || max < 0 || (max > 0 && !out)) return ORAC_ERR_PARAM;
  if (!ctx->d_ne) return ctx_fail(ctx, ORAC_ERR_STATE, "no schedule");
  CK(cudaSetDevice(ctx->device));
  long long n = 0;
  CK(cudaMemcpyAsync(&n, &ctx->d_ne->nrec, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (n_total) *n_total = n;
  const long long have = n < NE_REC_CAP ? n : NE_REC_CAP;
  const long long take = have < max ? have : max;
  std::vector<double> all(2 * (size_t)NE_REC_CAP);
  CK(cudaMemcpy(all.data(), ctx->d_ne->rec, sizeof(double) * 2 * NE_REC_CAP, cudaMemcpyDeviceToHost));
  for (long long k = 0; k < take; k++) {
    const long long r = (n - take + k) % NE_REC_CAP;
    out[2 * k] = all[2 * r];
    out[2 * k + 1] = all[2 * r + 1];
  }
  return ORAC_OK;
}

}  // extern "C"
