// C ABI, second part: fft_pme / do_pmesh_kspace (SPME) and the short-list
// routines fnb14, fnbgrp, ferrf, cself.
#include <cmath>

#include "common.cuh"

namespace {

__global__ void k_to_cart(int n, const double* __restrict__ s, double c11, double c12, double c13, double c22,
                          double c23, double c33, double* __restrict__ x) {
  pdl_enter();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double a = s[t], b = s[n + t], c = s[2 * n + t];
  x[t] = c11 * a + c12 * b + c13 * c;
  x[n + t] = c22 * b + c23 * c;
  x[2 * n + t] = c33 * c;
}

int ensure_host(orac_gpu_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->h_stage_bytes) return ORAC_OK;
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  ctx->h_stage = nullptr;
  ctx->h_stage_bytes = 0;
  CK(cudaMallocHost((void**)&ctx->h_stage, bytes));
  ctx->h_stage_bytes = bytes;
  return ORAC_OK;
}

int up_doubles(orac_gpu_ctx* ctx, double* dst, const double* const* srcs, int nsrc, size_t n) {
  if (int rc = ensure_host(ctx, sizeof(double) * n * nsrc)) return rc;
  for (int k = 0; k < nsrc; k++) memcpy(ctx->h_stage + k * n, srcs[k], sizeof(double) * n);
  CK(cudaMemcpyAsync(dst, ctx->h_stage, sizeof(double) * n * nsrc, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return ORAC_OK;
}

void recip_of(const double* oc, double* recip) {
  // src/fft_pme.f:47-51: recip(i,j) = 0.5 oc(j,i)
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) recip[i + 3 * j] = 0.5 * oc[j + 3 * i];
}

int ready(orac_gpu_ctx* ctx) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (!ctx->have_topo || !ctx->have_box || !ctx->have_ewald)
    return ctx_fail(ctx, ORAC_ERR_STATE, "topology, box and ewald parameters must be set");
  return ORAC_OK;
}

}  // namespace

static ApiScratch& scr(orac_gpu_ctx* ctx) { return ctx->api; }

template <typename T>
static int grow(orac_gpu_ctx* ctx, T** p, size_t* have, size_t n) {
  if (n <= *have && *p) return ORAC_OK;
  if (dev_alloc(ctx, p, n)) return ORAC_ERR_CUDA;
  *have = n;
  return ORAC_OK;
}

// device part of fft_pme: Cartesian conversion, SPME, molecular correction
int fft_pme_device(orac_gpu_ctx* ctx, const double* d_sxyz, const double* d_mol, double* d_f, double* d_eout) {
  ApiScratch& S = scr(ctx);
  const int N = ctx->N;
  if (grow(ctx, &S.cart, &S.cart_n, 3 * (size_t)N)) return ORAC_ERR_CUDA;
  const double* c = ctx->co;
  orac_launch(k_to_cart, (N + 255) / 256, 256, 0, ctx->stream, N, d_sxyz, c[0], c[3], c[6], c[4], c[7], c[8], S.cart);
  CKL();
  double recip[9];
  recip_of(ctx->oc, recip);
  const bool dq = ctx->variant == VAR_ALCH && ctx->d_dq && ctx->d_xtra;
  return pme_run(ctx, N, S.cart, ctx->pme_q(), recip, ctx->volume, ctx->alphal, d_f, d_eout, d_sxyz, d_mol, nullptr,
                 dq ? ctx->d_dq : nullptr, dq ? ctx->d_xtra + 5 : nullptr);
}

extern "C" {

int orac_gpu_fft_pme(orac_gpu_ctx* ctx, const double* xp, const double* yp, const double* zp, const double* xpcm,
                     const double* ypcm, const double* zpcm, double* eer, double* fpx, double* fpy, double* fpz,
                     double* stressc, int pressure) {
  if (int rc = ready(ctx)) return rc;
  if (!ctx->clewld) return ctx_fail(ctx, ORAC_ERR_STATE, "Ewald is off");
  CK(cudaSetDevice(ctx->device));
  ApiScratch& S = scr(ctx);
  const int N = ctx->N, P = ctx->P;
  const double* s3[3] = {xp, yp, zp};
  if (int rc = up_doubles(ctx, ctx->d_xyz, s3, 3, N)) return rc;
  const double* m3[3] = {xpcm, ypcm, zpcm};
  if (int rc = up_doubles(ctx, ctx->d_mol, m3, 3, P)) return rc;
  if (!S.eout && dev_alloc(ctx, &S.eout, 16)) return ORAC_ERR_CUDA;
  CK(cudaMemsetAsync(ctx->d_fout, 0, sizeof(double) * 3 * (size_t)N, ctx->stream));
  if (ctx->variant == VAR_ALCH && ctx->d_dq) {
    if (!ctx->d_xtra && dev_alloc(ctx, &ctx->d_xtra, 8)) return ORAC_ERR_CUDA;
    CK(cudaMemsetAsync(ctx->d_xtra + 5, 0, sizeof(double), ctx->stream));
  }
  if (int rc = fft_pme_device(ctx, ctx->d_xyz, ctx->d_mol, ctx->d_fout, S.eout)) return rc;
  if (int rc = ensure_host(ctx, sizeof(double) * (3 * (size_t)N + 16))) return rc;
  CK(cudaMemcpyAsync(ctx->h_stage, ctx->d_fout, sizeof(double) * 3 * (size_t)N, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_stage + 3 * (size_t)N, S.eout, sizeof(double) * 16, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double* f = ctx->h_stage;
  for (int a = 0; a < N; a++) {
    fpx[a] += f[a];
    fpy[a] += f[N + a];
    fpz[a] += f[2 * N + a];
  }
  const double* e = f + 3 * (size_t)N;
  *eer = 0.5 * e[0];
  ctx->pme_dwrk = 0.0;
  if (ctx->variant == VAR_ALCH && ctx->q0_differs) {
    // do_pmesh_alchemy (src/do_pmesh_alchemy.f90:66-87): a second grid of the
    // lambda0 charges gives eer0; the forces come from the lambda grid only
    double recip[9];
    recip_of(ctx->oc, recip);
    CK(cudaMemsetAsync(ctx->d_fout, 0, sizeof(double) * 3 * (size_t)N, ctx->stream));
    if (int rc = pme_run(ctx, N, S.cart, ctx->d_q0, recip, ctx->volume, ctx->alphal, ctx->d_fout, S.eout, nullptr,
                         nullptr))  // both already copied out above
      return rc;
    double e0 = 0.0;
    CK(cudaMemcpyAsync(&e0, S.eout, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->pme_dwrk = *eer - 0.5 * e0;
  }
  if (pressure) {
    // vir (symmetric, x0.5), src/scalar_sum.f:125-133; stressc(a,b) += -vir(a,b) + stc(a,b)
    const double vir[9] = {0.5 * e[1], 0.5 * e[4], 0.5 * e[5], 0.5 * e[4], 0.5 * e[2],
                           0.5 * e[6], 0.5 * e[5], 0.5 * e[6], 0.5 * e[3]};
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) stressc[a + 3 * b] += -vir[3 * a + b] + e[7 + 3 * a + b];
  }
  return ORAC_OK;
}

int orac_gpu_fft_pme_dev(orac_gpu_ctx* ctx, const double* xyz_scaled, const double* mol_scaled, double* fdev,
                         double* eer_dev, double* stress_dev) {
  (void)eer_dev;
  (void)stress_dev;
  if (int rc = ready(ctx)) return rc;
  CK(cudaSetDevice(ctx->device));
  ApiScratch& S = scr(ctx);
  if (!S.eout && dev_alloc(ctx, &S.eout, 16)) return ORAC_ERR_CUDA;
  return fft_pme_device(ctx, xyz_scaled, mol_scaled, fdev, eer_dev ? eer_dev : S.eout);
}

int orac_gpu_do_pmesh_kspace(orac_gpu_ctx* ctx, int numatoms, const double* x, const double* y, const double* z,
                             const double* charge, const double* recip, double volume, double ewald_coeff,
                             int order, int nfft1, int nfft2, int nfft3, double* eer, double* dx, double* dy,
                             double* dz, double* virial) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (numatoms <= 0) return ctx_fail(ctx, ORAC_ERR_PARAM, "numatoms = %d", numatoms);
  CK(cudaSetDevice(ctx->device));
  if (int rc = pme_setup(ctx, nfft1, nfft2, nfft3, order)) return rc;
  ApiScratch& S = scr(ctx);
  if (grow(ctx, &S.cart, &S.cart_n, 6 * (size_t)numatoms)) return ORAC_ERR_CUDA;
  if (grow(ctx, &S.q, &S.q_n, (size_t)numatoms)) return ORAC_ERR_CUDA;
  if (!S.eout && dev_alloc(ctx, &S.eout, 16)) return ORAC_ERR_CUDA;
  const double* s3[3] = {x, y, z};
  if (int rc = up_doubles(ctx, S.cart, s3, 3, numatoms)) return rc;
  const double* q1[1] = {charge};
  if (int rc = up_doubles(ctx, S.q, q1, 1, numatoms)) return rc;
  double* d_f = S.cart + 3 * (size_t)numatoms;
  CK(cudaMemsetAsync(d_f, 0, sizeof(double) * 3 * (size_t)numatoms, ctx->stream));
  const double saved_rk = ctx->rkcut;
  if (int rc = pme_run(ctx, numatoms, S.cart, S.q, recip, volume, ewald_coeff, d_f, S.eout, nullptr, nullptr))
    return rc;
  ctx->rkcut = saved_rk;
  if (int rc = ensure_host(ctx, sizeof(double) * (3 * (size_t)numatoms + 16))) return rc;
  CK(cudaMemcpyAsync(ctx->h_stage, d_f, sizeof(double) * 3 * (size_t)numatoms, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_stage + 3 * (size_t)numatoms, S.eout, sizeof(double) * 16, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double* f = ctx->h_stage;
  for (int a = 0; a < numatoms; a++) {
    dx[a] += f[a];
    dy[a] += f[numatoms + a];
    dz[a] += f[2 * (size_t)numatoms + a];
  }
  const double* e = f + 3 * (size_t)numatoms;
  *eer = 0.5 * e[0];
  const double vir[9] = {0.5 * e[1], 0.5 * e[4], 0.5 * e[5], 0.5 * e[4], 0.5 * e[2],
                         0.5 * e[6], 0.5 * e[5], 0.5 * e[6], 0.5 * e[3]};
  memcpy(virial, vir, sizeof(vir));  // symmetric: row- and column-major agree
  // restore the context's own grid for fft_pme
  if (ctx->clewld && ctx->nfft1 > 0) return pme_setup(ctx, ctx->nfft1, ctx->nfft2, ctx->nfft3, ctx->order);
  return ORAC_OK;
}

static int small_common(orac_gpu_ctx* ctx, int kind, const double* x0, const double* y0, const double* z0,
                        const int* pairs, int npairs, const int* ptype, int nptype, const double* t12,
                        const double* t6, int ntab, double fudge, double lj_fudge, int coul_mode, int forces,
                        double* fpx, double* fpy, double* fpz, double* e4) {
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  if (npairs < 0) return ctx_fail(ctx, ORAC_ERR_PARAM, "npairs < 0");
  CK(cudaSetDevice(ctx->device));
  const int N = ctx->N;
  for (int k = 0; k < 2 * npairs; k++)
    if (pairs[k] < 1 || pairs[k] > N) return ctx_fail(ctx, ORAC_ERR_PARAM, "pair atom index %d", pairs[k]);
  if (kind == 0)
    for (int k = 0; k < npairs; k++)
      if (ptype[k] < 1 || ptype[k] > ntab) return ctx_fail(ctx, ORAC_ERR_PARAM, "type14 index %d", ptype[k]);
  ApiScratch& S = scr(ctx);
  if (grow(ctx, &S.cart, &S.cart_n, 6 * (size_t)N)) return ORAC_ERR_CUDA;
  if (grow(ctx, &S.ipairs, &S.ipairs_n, 2 * (size_t)npairs + 2)) return ORAC_ERR_CUDA;
  if (grow(ctx, &S.itype, &S.itype_n, (size_t)(nptype > 0 ? nptype : 1))) return ORAC_ERR_CUDA;
  if (ntab > 0 && (ntab > (int)S.tab_n || !S.t12)) {
    if (dev_alloc(ctx, &S.t12, ntab) || dev_alloc(ctx, &S.t6, ntab)) return ORAC_ERR_CUDA;
    S.tab_n = ntab;
  }
  if (!S.e4 && dev_alloc(ctx, &S.e4, 4)) return ORAC_ERR_CUDA;
  if (!S.ss) {
    if (dev_alloc(ctx, &S.ss, N)) return ORAC_ERR_CUDA;
    CK(cudaMemcpy(S.ss, ctx->h_ss.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  }
  const double* s3[3] = {x0, y0, z0};
  if (int rc = up_doubles(ctx, S.cart, s3, 3, N)) return rc;
  double* d_f = S.cart + 3 * (size_t)N;
  CK(cudaMemsetAsync(d_f, 0, sizeof(double) * 3 * (size_t)N, ctx->stream));
  CK(cudaMemsetAsync(S.e4, 0, sizeof(double) * 4, ctx->stream));
  if (npairs > 0) {
    CK(cudaMemcpyAsync(S.ipairs, pairs, sizeof(int) * 2 * (size_t)npairs, cudaMemcpyHostToDevice, ctx->stream));
    if (nptype > 0)
      CK(cudaMemcpyAsync(S.itype, ptype, sizeof(int) * (size_t)nptype, cudaMemcpyHostToDevice, ctx->stream));
    if (ntab > 0) {
      CK(cudaMemcpyAsync(S.t12, t12, sizeof(double) * ntab, cudaMemcpyHostToDevice, ctx->stream));
      CK(cudaMemcpyAsync(S.t6, t6, sizeof(double) * ntab, cudaMemcpyHostToDevice, ctx->stream));
    }
    if (int rc = small_launch(ctx, kind, S.cart, S.ipairs, S.itype, npairs, S.t12, S.t6, fudge, lj_fudge, coul_mode,
                              forces, d_f, S.e4, S.ss))
      return rc;
  }
  if (int rc = ensure_host(ctx, sizeof(double) * (3 * (size_t)N + 4))) return rc;
  CK(cudaMemcpyAsync(ctx->h_stage, d_f, sizeof(double) * 3 * (size_t)N, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_stage + 3 * (size_t)N, S.e4, sizeof(double) * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (forces)
    for (int a = 0; a < N; a++) {
      fpx[a] += ctx->h_stage[a];
      fpy[a] += ctx->h_stage[N + a];
      fpz[a] += ctx->h_stage[2 * (size_t)N + a];
    }
  memcpy(e4, ctx->h_stage + 3 * (size_t)N, 4 * sizeof(double));
  return ORAC_OK;
}

int orac_gpu_fnb14(orac_gpu_ctx* ctx, const double* xp0, const double* yp0, const double* zp0, int cut,
                   const int* int14, int int14p, const int* type14, const double* ecc1412, const double* ecc146,
                   int ntab, double fudge, double lj_fudge, double* fpx, double* fpy, double* fpz, double* ue) {
  // src/fnb14.f:86: bare Coulomb unless (ewald and cut)
  const int coul = (ctx && ctx->clewld && cut) ? 1 : 0;
  return small_common(ctx, 0, xp0, yp0, zp0, int14, int14p, type14, int14p, ecc1412, ecc146, ntab, fudge, lj_fudge,
                      coul, 1, fpx, fpy, fpz, ue);
}

int orac_gpu_fnbgrp(orac_gpu_ctx* ctx, const double* xp0, const double* yp0, const double* zp0, const int* ingrp,
                    int ingrpp, double* fpx, double* fpy, double* fpz, double* ue) {
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  // fnbgrp indexes ecc12/ecc6 by the triangular index of the two nbtypes
  // (src/fnbgrp.f:100-103) and takes Ewald from clewld
  return small_common(ctx, 1, xp0, yp0, zp0, ingrp, ingrpp, ctx->h_nbtype.data(), ctx->N, ctx->h_ecc12.data(),
                      ctx->h_ecc6.data(), (int)ctx->h_ecc12.size(), 1.0, 1.0, ctx->clewld, 1, fpx, fpy, fpz, ue);
}

int orac_gpu_ferrf(orac_gpu_ctx* ctx, double fudge, const double* x0, const double* y0, const double* z0, int iz,
                   const int* list, int nlist, double* fs, double* fpx, double* fpy, double* fpz) {
  double e4[4];
  const int rc = small_common(ctx, 2, x0, y0, z0, list, nlist, nullptr, 0, nullptr, nullptr, 0, fudge, 1.0, 1,
                              iz == 1 ? 1 : 0, fpx, fpy, fpz, e4);
  if (rc) return rc;
  fs[0] = e4[0];
  fs[1] = e4[1];
  return ORAC_OK;
}

int orac_gpu_cself(orac_gpu_ctx* ctx, double kcut, double* self_slt, double* self_slv) {
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  CK(cudaSetDevice(ctx->device));
  ApiScratch& S = scr(ctx);
  if (!S.e4 && dev_alloc(ctx, &S.e4, 4)) return ORAC_ERR_CUDA;
  if (!S.ss) {
    if (dev_alloc(ctx, &S.ss, ctx->N)) return ORAC_ERR_CUDA;
    CK(cudaMemcpy(S.ss, ctx->h_ss.data(), sizeof(int) * ctx->N, cudaMemcpyHostToDevice));
  }
  CK(cudaMemsetAsync(S.e4, 0, sizeof(double) * 4, ctx->stream));
  if (int rc = self_launch(ctx, S.ss, S.e4)) return rc;
  double e[2];
  CK(cudaMemcpyAsync(e, S.e4, sizeof(double) * 2, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // src/cself.f:51-57
  const double alphar = kcut / (2.0 * ctx->alphal);
  const double qt = 1.0 / (1.0 + 0.3275911 * alphar);
  const double erfcst =
      ((((1.0614054 * qt - 1.453152) * qt + 1.4214137) * qt - 0.28449674) * qt + 0.2548296) * qt *
      std::exp(-alphar * alphar);
  const double pi = 4.0 * std::atan(1.0);
  *self_slt = -e[0] * ctx->alphal / std::sqrt(pi) * (1.0 - erfcst);
  *self_slv = -e[1] * ctx->alphal / std::sqrt(pi) * (1.0 - erfcst);
  return ORAC_OK;
}

}  // extern "C"
