// C ABI of the intramolecular path: the bonded terms and pair lists of
// mts_intra_n0 (src/mts_intra_n0.f) and mts_intra_n1 (src/mts_intra_n1.f).
// ORAC keeps these in module arrays (lstrtch, lbndg, ltor, litr, int14,
// ingrp, int13 with their parameter tables); here they are uploaded once.
#include <cmath>

#include "common.cuh"

namespace {

template <typename T>
int upload(orac_gpu_ctx* ctx, T** dst, const std::vector<T>& v) {
  if (*dst) dev_free(ctx, *dst);
  *dst = nullptr;
  if (v.empty()) return ORAC_OK;
  if (dev_alloc(ctx, dst, v.size())) return ORAC_ERR_CUDA;
  CK(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return ORAC_OK;
}

int check_atoms(orac_gpu_ctx* ctx, const int* l, int n, int w, const char* what) {
  for (int k = 0; k < n * w; k++)
    if (l[k] < 1 || l[k] > ctx->N) return ctx_fail(ctx, ORAC_ERR_PARAM, "%s: atom index %d out of 1..%d", what, l[k], ctx->N);
  return ORAC_OK;
}

int ensure_ss(orac_gpu_ctx* ctx) {
  BondedDev& B = ctx->bd;
  if (B.ss) return ORAC_OK;
  return upload(ctx, &B.ss, ctx->h_ss);
}

int up_pairs(orac_gpu_ctx* ctx, int** dst, const int* p, int n) {
  std::vector<int> v(p, p + 2 * (size_t)n);
  return upload(ctx, dst, v);
}

// host staging of Cartesian coordinates and the force / energy readback
struct Stage {
  double* x = nullptr;
  double* f = nullptr;
  double* e = nullptr;
};

int stage_in(orac_gpu_ctx* ctx, const double* x, const double* y, const double* z, Stage* S) {
  const int N = ctx->N;
  BondedDev& B = ctx->bd;
  if (!B.xs && (dev_alloc(ctx, &B.xs, 6 * (size_t)N + 16))) return ORAC_ERR_CUDA;
  if (!ctx->h_stage || ctx->h_stage_bytes < sizeof(double) * (3 * (size_t)N + 16)) {
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    ctx->h_stage = nullptr;
    ctx->h_stage_bytes = 0;
    CK(cudaMallocHost((void**)&ctx->h_stage, sizeof(double) * (3 * (size_t)N + 16)));
    ctx->h_stage_bytes = sizeof(double) * (3 * (size_t)N + 16);
  }
  memcpy(ctx->h_stage, x, sizeof(double) * N);
  memcpy(ctx->h_stage + N, y, sizeof(double) * N);
  memcpy(ctx->h_stage + 2 * N, z, sizeof(double) * N);
  S->x = B.xs;
  S->f = B.xs + 3 * (size_t)N;
  S->e = B.xs + 6 * (size_t)N;
  CK(cudaMemcpyAsync(S->x, ctx->h_stage, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(S->f, 0, sizeof(double) * (3 * (size_t)N + 16), ctx->stream));
  return ORAC_OK;
}

int stage_out(orac_gpu_ctx* ctx, double* fpx, double* fpy, double* fpz, double* e, int ne) {
  const int N = ctx->N;
  const double* src = ctx->bd.xs + 3 * (size_t)N;  // forces, then the energies
  CK(cudaMemcpyAsync(ctx->h_stage, src, sizeof(double) * (3 * (size_t)N + ne), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int a = 0; a < N; a++) {
    fpx[a] += ctx->h_stage[a];
    fpy[a] += ctx->h_stage[N + a];
    fpz[a] += ctx->h_stage[2 * N + a];
  }
  for (int k = 0; k < ne; k++) e[k] = ctx->h_stage[3 * N + k];
  return ORAC_OK;
}

}  // namespace

void bonded_free(orac_gpu_ctx* ctx) {
  BondedDev& B = ctx->bd;
  void* p[] = {B.bij, B.bpar, B.aijk, B.apot, B.tijkl, B.tpar, B.iijkl, B.ipar, B.ss, B.p14, B.t14,
               B.e1412, B.e146, B.pgrp, B.p13, B.pbond, B.pcn, B.nbt, B.e12, B.e6, B.xs};
  for (void* q : p)
    if (q) dev_free(ctx, q);
  ctx->bd = BondedDev();
}

int bonded_set_constraints(orac_gpu_ctx* ctx, const int* cnst, int ncnst) {
  ctx->bd.ncn = ncnst;
  // the erf correction kernel reads ss_index of every listed pair
  if (int rc = ensure_ss(ctx)) return rc;
  return up_pairs(ctx, &ctx->bd.pcn, cnst, ncnst);
}

extern "C" {

int orac_gpu_set_bonded(orac_gpu_ctx* ctx, int nb, const int* lbnd, const double* r0, const double* kb, int nbend,
                        const int* lbndg, const double* bendpot, int nt, const int* ltor, const double* tpota,
                        const double* tpotb, int nit, const int* litr, const double* ipota, const double* ipotb,
                        const double* ipotc) {
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  if (nb < 0 || nbend < 0 || nt < 0 || nit < 0) return ctx_fail(ctx, ORAC_ERR_PARAM, "negative term count");
  CK(cudaSetDevice(ctx->device));
  if (int rc = check_atoms(ctx, lbnd, nb, 2, "lbnd")) return rc;
  if (int rc = check_atoms(ctx, lbndg, nbend, 3, "lbndg")) return rc;
  if (int rc = check_atoms(ctx, ltor, nt, 4, "ltor")) return rc;
  if (int rc = check_atoms(ctx, litr, nit, 4, "litr")) return rc;
  BondedDev& B = ctx->bd;
  // intramolecular-level membership of the atoms (k_drift skips the N0/N1
  // accumulators of small molecules with none)
  ctx->h_intra_b.assign(ctx->N, 0);
  auto mark = [&](const int* l, int n, int w, unsigned char bit) {
    for (int k = 0; k < n * w; k++) ctx->h_intra_b[l[k] - 1] |= bit;
  };
  mark(lbnd, nb, 2, 1);
  mark(lbndg, nbend, 3, 1);
  mark(litr, nit, 4, 1);
  mark(ltor, nt, 4, 2);
  std::vector<int2> bij(nb);
  std::vector<double2> bpar(nb);
  for (int k = 0; k < nb; k++) {
    bij[k] = make_int2(lbnd[2 * k] - 1, lbnd[2 * k + 1] - 1);
    bpar[k] = make_double2(r0[k], kb[k]);
  }
  std::vector<int4> aijk(nbend);
  std::vector<double> apot(bendpot, bendpot + 7 * (size_t)nbend);
  for (int k = 0; k < nbend; k++) aijk[k] = make_int4(lbndg[3 * k] - 1, lbndg[3 * k + 1] - 1, lbndg[3 * k + 2] - 1, 0);
  std::vector<int4> tijkl(nt), iijkl(nit);
  std::vector<double2> tpar(nt);
  std::vector<double4> ipar(nit);
  for (int k = 0; k < nt; k++) {
    tijkl[k] = make_int4(ltor[4 * k] - 1, ltor[4 * k + 1] - 1, ltor[4 * k + 2] - 1, ltor[4 * k + 3] - 1);
    tpar[k] = make_double2(tpota[k], tpotb[k]);
  }
  for (int k = 0; k < nit; k++) {
    iijkl[k] = make_int4(litr[4 * k] - 1, litr[4 * k + 1] - 1, litr[4 * k + 2] - 1, litr[4 * k + 3] - 1);
    ipar[k] = make_double4(ipota[k], ipotb[k], ipotc[k], 0.0);
  }
  if (upload(ctx, &B.bij, bij) || upload(ctx, &B.bpar, bpar) || upload(ctx, &B.aijk, aijk) ||
      upload(ctx, &B.apot, apot) || upload(ctx, &B.tijkl, tijkl) || upload(ctx, &B.tpar, tpar) ||
      upload(ctx, &B.iijkl, iijkl) || upload(ctx, &B.ipar, ipar) || ensure_ss(ctx))
    return ORAC_ERR_CUDA;
  B.nb = nb;
  B.nbend = nbend;
  B.nt = nt;
  B.nit = nit;
  // the bonds are also the first list of the erf corrections
  return up_pairs(ctx, &B.pbond, lbnd, nb);
}

int orac_gpu_set_intra_pairs(orac_gpu_ctx* ctx, int n14, const int* int14, const int* type14, const double* ecc1412,
                             const double* ecc146, int ntab14, double fudge, double lj_fudge, int ningrp,
                             const int* ingrp, int n13, const int* int13) {
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  if (n14 < 0 || ningrp < 0 || n13 < 0) return ctx_fail(ctx, ORAC_ERR_PARAM, "negative pair count");
  CK(cudaSetDevice(ctx->device));
  if (int rc = check_atoms(ctx, int14, n14, 2, "int14")) return rc;
  if (int rc = check_atoms(ctx, ingrp, ningrp, 2, "ingrp")) return rc;
  if (int rc = check_atoms(ctx, int13, n13, 2, "int13")) return rc;
  for (int k = 0; k < n14; k++)
    if (type14[k] < 1 || type14[k] > ntab14) return ctx_fail(ctx, ORAC_ERR_PARAM, "type14 %d", type14[k]);
  BondedDev& B = ctx->bd;
  ctx->h_intra_p.assign(ctx->N, 0);
  for (int k = 0; k < 2 * n14; k++) ctx->h_intra_p[int14[k] - 1] |= 2;
  for (int k = 0; k < 2 * ningrp; k++) ctx->h_intra_p[ingrp[k] - 1] |= 2;
  std::vector<int> t14(type14, type14 + n14);
  std::vector<double> e12(ecc1412, ecc1412 + ntab14), e6(ecc146, ecc146 + ntab14);
  std::vector<double> l12(ctx->h_ecc12), l6(ctx->h_ecc6);
  if (up_pairs(ctx, &B.p14, int14, n14) || upload(ctx, &B.t14, t14) || upload(ctx, &B.e1412, e12) ||
      upload(ctx, &B.e146, e6) || up_pairs(ctx, &B.pgrp, ingrp, ningrp) || up_pairs(ctx, &B.p13, int13, n13) ||
      upload(ctx, &B.nbt, ctx->h_nbtype) || upload(ctx, &B.e12, l12) || upload(ctx, &B.e6, l6) || ensure_ss(ctx))
    return ORAC_ERR_CUDA;
  B.n14 = n14;
  B.ntab14 = ntab14;
  B.fudge = fudge;
  B.lj_fudge = lj_fudge;
  B.ningrp = ningrp;
  B.n13 = n13;
  B.have_pairs = true;
  return ORAC_OK;
}

int orac_gpu_mts_intra_n0(orac_gpu_ctx* ctx, const double* x, const double* y, const double* z, double* fpx,
                          double* fpy, double* fpz, double* energies) {
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  CK(cudaSetDevice(ctx->device));
  Stage S;
  if (int rc = stage_in(ctx, x, y, z, &S)) return rc;
  if (int rc = bonded_launch(ctx, BK_BOND | BK_BEND | BK_ITORS, S.x, S.f, nullptr, S.e)) return rc;
  double e[8];
  if (int rc = stage_out(ctx, fpx, fpy, fpz, e, 8)) return rc;
  // ubond, uslvbon, ubend, uslvben, uitors, uslvitor
  const double out[6] = {e[0], e[1], e[2], e[3], e[6], e[7]};
  memcpy(energies, out, sizeof(out));
  return ORAC_OK;
}

int orac_gpu_mts_intra_n1(orac_gpu_ctx* ctx, const double* x, const double* y, const double* z, double* fpx,
                          double* fpy, double* fpz, double* energies) {
  if (!ctx || !ctx->have_topo) return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "topology not set") : ORAC_ERR_PARAM;
  CK(cudaSetDevice(ctx->device));
  Stage S;
  if (int rc = stage_in(ctx, x, y, z, &S)) return rc;
  if (int rc = bonded_launch(ctx, BK_TORS, S.x, S.f, nullptr, S.e)) return rc;
  const BondedDev& B = ctx->bd;
  if (B.have_pairs) {
    const int coul = ctx->clewld ? 1 : 0;
    if (int rc = small_launch_x(ctx, 0, S.x, B.p14, B.t14, B.n14, B.e1412, B.e146, B.fudge, B.lj_fudge, coul, 1, S.f,
                                S.e + 8, B.ss, nullptr, nullptr))
      return rc;
    if (int rc = small_launch_x(ctx, 1, S.x, B.pgrp, B.nbt, B.ningrp, B.e12, B.e6, 1.0, 1.0, coul, 1, S.f, S.e + 12,
                                B.ss, nullptr, nullptr))
      return rc;
  }
  double e[16];
  if (int rc = stage_out(ctx, fpx, fpy, fpz, e, 16)) return rc;
  // uptors, uslvtor, 1-4 (LJ slt, LJ slv, Coul slt, Coul slv), intra-group (same)
  const double out[10] = {e[4], e[5], e[8], e[9], e[10], e[11], e[12], e[13], e[14], e[15]};
  memcpy(energies, out, sizeof(out));
  return ORAC_OK;
}

}  // extern "C"
