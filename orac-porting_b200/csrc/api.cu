// C ABI of liborac_gpu.so (declared in include/orac_gpu.h): context life
// cycle, upload of ORAC's module globals, and the host side of the
// mts_forces / lc_list / fft_pme / do_pmesh_kspace / fnb14 / fnbgrp / ferrf /
// cself entry points.  Host arrays are staged through pinned memory; every
// computation runs on the context's stream.
#include <cmath>
#include <cstdlib>
#include <string>

#include "common.cuh"

int ctx_fail(orac_gpu_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(c->err, sizeof(c->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

namespace {

constexpr double AS_A1 = 0.2548296, AS_A2 = -0.28449674, AS_A3 = 1.4214137;
constexpr double AS_A4 = -1.453152, AS_A5 = 1.0614054, AS_QP = 0.3275911;

double erfc_as(double x) {
  const double qt = 1.0 / (1.0 + AS_QP * x);
  return ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * std::exp(-x * x);
}

int ensure_stage(orac_gpu_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->h_stage_bytes) return ORAC_OK;
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  ctx->h_stage = nullptr;
  ctx->h_stage_bytes = 0;
  CK(cudaMallocHost((void**)&ctx->h_stage, bytes));
  ctx->h_stage_bytes = bytes;
  return ORAC_OK;
}

// Copy k host arrays of n doubles each into consecutive device memory.
int upload3(orac_gpu_ctx* ctx, double* dst, int n, const double* a, const double* b, const double* c) {
  if (int rc = ensure_stage(ctx, sizeof(double) * 3 * (size_t)n)) return rc;
  memcpy(ctx->h_stage, a, sizeof(double) * n);
  memcpy(ctx->h_stage + n, b, sizeof(double) * n);
  memcpy(ctx->h_stage + 2 * (size_t)n, c, sizeof(double) * n);
  CK(cudaMemcpyAsync(dst, ctx->h_stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));  // staging buffer is reused
  return ORAC_OK;
}

__global__ void k_shell_out(const double* __restrict__ acc, int forces_on, double* __restrict__ e,
                            double* __restrict__ stress) {
  pdl_enter();
  const int t = threadIdx.x;
  if (e && t < 8) {
    // ORAC argument order: ucns ucos virs virsp ucnp ucop ucnsp ucosp
    const int src[8] = {ACC_CONF + 2, ACC_COUL + 2, -1, -1, ACC_CONF + 0, ACC_COUL + 0, ACC_CONF + 1, ACC_COUL + 1};
    e[t] = (forces_on && src[t] >= 0) ? acc[src[t]] : 0.0;
  }
  if (stress && t < 9) {
    const int i = t / 3, j = t % 3;  // stress(i,j) column-major
    stress[i + 3 * j] = forces_on ? acc[ACC_STR + t] + acc[ACC_VIMG + t] : 0.0;
  }
}

struct ShellSel {
  double ro, ri, rto, rti, rni;
  int iz;
  int in, out;  // list indices
};

// src/mts_forces.f:57-93
int select_shell(orac_gpu_ctx* ctx, const ShellRadii& r, char rshell, ShellSel* s) {
  switch (rshell) {
    case 'u':
      *s = {r.rcuth, r.rcuth, 0.0, r.rtolh, r.rneih, 0, -1, 0};
      return ORAC_OK;
    case 'h':
      *s = {r.rcuth, r.rcutl, r.rtolh, r.rtoll, r.rneil, r.rneih < 1e-10 ? 0 : 1, 0, 1};
      return ORAC_OK;
    case 'l':
      *s = {r.rcutl, r.rcutm, r.rtoll, r.rtolm, r.rneim, 1, 1, 2};
      return ORAC_OK;
    case 'm':
      *s = {r.rcutm, 0.0, r.rtolm, 0.0, 0.0, 1, 2, -1};
      return ORAC_OK;
    default:
      return ctx_fail(ctx, ORAC_ERR_PARAM, "unknown shell '%c'", rshell);
  }
}

int check_ready(orac_gpu_ctx* ctx) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (!ctx->have_topo) return ctx_fail(ctx, ORAC_ERR_STATE, "topology not set");
  if (!ctx->have_box) return ctx_fail(ctx, ORAC_ERR_STATE, "box not set");
  if (!ctx->have_shells) return ctx_fail(ctx, ORAC_ERR_STATE, "shells not set");
  if (!ctx->have_ewald) return ctx_fail(ctx, ORAC_ERR_STATE, "ewald parameters not set");
  return ORAC_OK;
}

}  // namespace

// Shell evaluation on device-resident coordinates (used by both ABIs).
int shell_run(orac_gpu_ctx* ctx, char rshell, const double* d_xyz, const double* d_grp, const double* d_mol,
              double* d_f, double* d_e, double* d_stress, int energy) {
  return shell_run_r(ctx, rshell, ctx->sh, d_xyz, d_grp, d_mol, d_f, d_e, d_stress,
                     SH_STRESS | (energy ? SH_ENERGY : 0));
}

int shell_run_r(orac_gpu_ctx* ctx, char rshell, const ShellRadii& radii, const double* d_xyz, const double* d_grp,
                const double* d_mol, double* d_f, double* d_e, double* d_stress, int flags) {
  ShellSel s;
  if (int rc = select_shell(ctx, radii, rshell, &s)) return rc;
  if (rshell == 'u') {
    if (ctx->ncx > 0)
      return ctx_fail(ctx, ORAC_ERR_PARAM, "'u' update is for runs without LINKED_CELL; use orac_gpu_lc_list");
    if (d_grp != ctx->d_grp)
      CK(cudaMemcpyAsync(ctx->d_grp, d_grp, sizeof(double) * 3 * ctx->G, cudaMemcpyDeviceToDevice, ctx->stream));
    if (int rc = list_build_allpairs(ctx, s.ri + s.rti + s.rni, &ctx->lists[0])) return rc;
    if (d_e) CK(cudaMemsetAsync(d_e, 0, 8 * sizeof(double), ctx->stream));
    if (d_stress) CK(cudaMemsetAsync(d_stress, 0, 9 * sizeof(double), ctx->stream));
    return ORAC_OK;
  }
  GList& Lin = ctx->lists[s.in];
  if (!Lin.valid)
    return ctx_fail(ctx, ORAC_ERR_STATE, "shell '%c' called before its neighbour list was built", rshell);
  // radii of src/force.f:145-167 (rinn0 takes rtolinn before its reset)
  const double rinn = s.ri, rout = s.ro;
  double rtolinn = s.rti;
  const double rtolout = s.rto;
  const double rinn0 = rinn + rtolinn;
  if (rinn < 1e-5) rtolinn = 0.0;
  const double rout0 = rout + rtolout;
  PairArgs a;
  memset(&a, 0, sizeof(a));
  a.gpos = ctx->d_gpos;
  a.gmeta = ctx->d_gmeta;
  a.aoff = ctx->d_aoff;
  a.atype = ctx->d_atype;
  a.apm = ctx->d_apm;
  a.lj = ctx->d_lj;
  a.ntype = ctx->ntype;
  a.ngrp = ctx->G;
  a.c11 = ctx->co[0];
  a.c12 = ctx->co[3];
  a.c13 = ctx->co[6];
  a.c22 = ctx->co[4];
  a.c23 = ctx->co[7];
  a.c33 = ctx->co[8];
  a.r2inn = rinn * rinn;
  a.r2out = rout * rout;
  a.rinn0 = rinn0;
  a.r2inn0 = rinn0 * rinn0;
  a.rout0 = rout0;
  a.r2out0 = rout0 * rout0;
  a.r2neigh = (rinn0 + s.rni) * (rinn0 + s.rni);
  a.arsout1 = rout0 - 3.0 * rout;
  a.arsout2 = rtolout * rtolout * rtolout;
  a.arsinn1 = rinn0 - 3.0 * rinn;
  a.arsinn2 = rtolinn * rtolinn * rtolinn;
  a.iarsout2 = a.arsout2 > 0.0 ? (float)(1.0 / a.arsout2) : 0.0f;
  a.iarsinn2 = a.arsinn2 > 0.0 ? (float)(1.0 / a.arsinn2) : 0.0f;
  a.diarsout2 = a.arsout2 > 0.0 ? 1.0 / a.arsout2 : 0.0;
  a.diarsinn2 = a.arsinn2 > 0.0 ? 1.0 / a.arsinn2 : 0.0;
  a.alphal = (float)ctx->alphal;
  a.alphad = ctx->alphal;
  a.ljd = ctx->d_ljd;
  a.qd = ctx->d_aqd;
  a.twrtpi = (float)(2.0 / std::sqrt(4.0 * std::atan(1.0)));
  a.forces_on = (s.iz == 1 && rinn0 < rout) ? 1 : 0;  // src/force.f:288,848
  a.next_on = (a.r2inn > 1.0e-5 && s.out >= 0 && !(flags & SH_NO_NEXT)) ? 1 : 0;  // src/force.f:279,337
  a.lskip = ctx->clewld ? (erfc_as(ctx->alphal * rinn) < 10.0e-4) : 1;  // decide_force
  a.ewald = ctx->clewld;
  a.off = Lin.off;
  a.cnt = Lin.cnt;
  a.lj_ = Lin.j;
  a.lmask = Lin.mask;
  if (a.next_on) {
    GList& Lout = ctx->lists[s.out];
    a.cnt_out = Lout.cnt;
    a.j_out = Lout.j;
    a.mask_out = Lout.mask;
  }
  a.ffix = ctx->d_ffix;
  a.acc = ctx->d_acc;
  a.natom = ctx->N;
  a.wcnt = ctx->d_wcnt;
  variant_fill(ctx, &a);
  // launch configuration: the tuned one, or the mode's default -- the
  // innermost shell's rows hold about a dozen groups: beside other contexts
  // half a warp each (fewer instructions per row) and 8 blocks per SM, alone
  // a warp each (twice the warps to hide one launch's latency) and 6
  if (rshell == 'm')
    a.lpg = ctx->tune_lpg_m ? ctx->tune_lpg_m : (ctx->shared_device ? 16 : 32);
  else
    a.lpg = ctx->tune_lpg_lh ? ctx->tune_lpg_lh : 32;
  a.minb = ctx->tune_minb ? ctx->tune_minb : (ctx->shared_device ? 8 : 6);
  // a row's entries split between two warps: only where twice the warps
  // still fit in one wave (a launch of the M shell, which writes no next
  // list, on a system of at most 1,024 groups); beyond that the second
  // wave costs more than the shorter chains save
  a.split = (rshell == 'm' && a.lpg == 32 && !a.next_on && !ctx->shared_device && ctx->G <= 1024) ? 2 : 1;
  const bool want_e = (flags & SH_ENERGY) && d_e, want_s = (flags & SH_STRESS) && d_stress;
  a.energy = want_e ? 1 : 0;
  a.stress = want_s ? 1 : 0;
  // the forces-only build sums force_alchemy's dwrk where a schedule asks
  a.dwrk = (a.variant == VAR_ALCH && !want_e && !want_s) ? ctx->pair_dwrk : nullptr;
  if (flags & SH_FIXED_OUT) a.ffix = reinterpret_cast<unsigned long long*>(d_f);
  if (want_e || want_s) CK(cudaMemsetAsync(ctx->d_acc, 0, ACC_N * sizeof(double), ctx->stream));
  if (!(flags & SH_PREPPED))
    if (int rc = prep_launch(ctx, d_xyz, d_grp)) return rc;
  if (int rc = pair_launch(ctx, a, ctx->maxg)) return rc;
  if (a.forces_on && !(flags & SH_FIXED_OUT))
    if (int rc = finalize_launch(ctx, d_mol, d_f, want_s ? 1 : 0)) return rc;
  if (want_e || want_s) {
    orac_launch(k_shell_out, 1, 32, 0, ctx->stream, ctx->d_acc, a.forces_on, want_e ? d_e : nullptr,
                                           want_s ? d_stress : nullptr);
    CKL();
  }
  if (want_e && ctx->variant != VAR_STD)
    if (int rc = variant_out_launch(ctx, a.forces_on)) return rc;
  if (a.next_on) ctx->lists[s.out].valid = true;
  return ORAC_OK;
}

// --------------------------------------------------------------------- ABI

extern "C" {

const char* orac_gpu_version(void) { return "orac_gpu 0.1 (sm_100a)"; }

const char* orac_gpu_last_error(const orac_gpu_ctx* ctx) { return ctx ? ctx->err : "null context"; }

int orac_gpu_create(int device, orac_gpu_ctx** out) {
  if (!out) return ORAC_ERR_PARAM;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ORAC_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return ORAC_ERR_PARAM;
  orac_gpu_ctx* ctx = new orac_gpu_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return ORAC_ERR_CUDA;
  }
  if (dev_alloc(ctx, &ctx->d_acc, ACC_N) || dev_alloc(ctx, &ctx->d_red, 64) || dev_alloc(ctx, &ctx->d_total, 4) ||
      dev_alloc(ctx, &ctx->d_flag, 4) || dev_alloc(ctx, &ctx->d_wcnt, 4) ||
      cudaMemset(ctx->d_wcnt, 0, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    orac_gpu_destroy(ctx);
    return ORAC_ERR_CUDA;
  }
  *out = ctx;
  return ORAC_OK;
}

int orac_gpu_destroy(orac_gpu_ctx* ctx) {
  if (!ctx) return ORAC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  md_destroy(ctx);
  void* ptrs[] = {ctx->d_gmeta, ctx->d_atype, ctx->d_apm, ctx->d_aq, ctx->d_aqd, ctx->d_amol, ctx->d_agrp,
                  ctx->d_gmol, ctx->d_amassinf, ctx->d_lj, ctx->d_ljd, ctx->d_exoff, ctx->d_exj, ctx->d_xyz, ctx->d_grp,
                  ctx->d_mol, ctx->d_gpos, ctx->d_aoff, ctx->d_ffix, ctx->d_acc, ctx->d_fout, ctx->d_red,
                  ctx->d_scan_tmp, ctx->d_total, ctx->d_flag, ctx->d_cell_of, ctx->d_cell_cnt, ctx->d_cell_start,
                  ctx->d_cell_grp, ctx->d_stencil, ctx->pme.tw1, ctx->pme.tw2, ctx->pme.tw3, ctx->pme.bsp1,
                  ctx->pme.bsp2, ctx->pme.bsp3, ctx->pme.qfix, ctx->pme.cgrid, ctx->pme.rgrid, ctx->pme.theta};
  for (void* p : ptrs)
    if (p) dev_free(ctx, p);
  void* aps[] = {ctx->api.cart, ctx->api.eout, ctx->api.ipairs, ctx->api.itype, ctx->api.t12,
                 ctx->api.t6,   ctx->api.ss,   ctx->api.e4,     ctx->api.q};
  for (void* p : aps)
    if (p) dev_free(ctx, p);
  if (ctx->d_wcnt) dev_free(ctx, ctx->d_wcnt);
  variant_free(ctx);
  bonded_free(ctx);
  for (auto& e : ctx->prof_ev) cudaEventDestroy(e);
  for (int q = 0; q < 3; q++) {
    if (q == 0 && ctx->lists[q].off) dev_free(ctx, ctx->lists[q].off);
    if (ctx->lists[q].cnt) dev_free(ctx, ctx->lists[q].cnt);
    if (ctx->lists[q].j) dev_free(ctx, ctx->lists[q].j);
    if (ctx->lists[q].mask) dev_free(ctx, ctx->lists[q].mask);
  }
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return ORAC_OK;
}

int orac_gpu_footprint(orac_gpu_ctx* ctx, int64_t* bytes) {
  if (!ctx || !bytes) return ORAC_ERR_PARAM;
  *bytes = (int64_t)ctx->dmem_bytes;
  return ORAC_OK;
}

int orac_gpu_set_topology(orac_gpu_ctx* ctx, int ntap, int ngrp, int nprot, const int* grppt, const int* atomp,
                          const int* atomg, const int* ss_index, const double* chrge, const int* nbtype, int ntype,
                          const int* type_table, const double* ecc12, const double* ecc6, const double* mass,
                          const double* pmass, double massinfty, const int* mapnl, int64_t nmapnl) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (ntap <= 0 || ngrp <= 0 || nprot <= 0 || ntype <= 0)
    return ctx_fail(ctx, ORAC_ERR_PARAM, "bad sizes ntap=%d ngrp=%d nprot=%d ntype=%d", ntap, ngrp, nprot, ntype);
  CK(cudaSetDevice(ctx->device));
  const int N = ntap, G = ngrp, P = nprot;
  std::vector<int2> gmeta(G);
  std::vector<int> gmol(G), agrp(N), amol(N), atype(N);
  std::vector<float> apm(N), aq(N);
  std::vector<unsigned char> minf(N);
  int maxg = 0;
  int prev_last = 0;
  for (int g = 0; g < G; g++) {
    const int a0 = grppt[2 * g] - 1, a1 = grppt[2 * g + 1] - 1;
    if (a0 != prev_last || a1 < a0 || a1 >= N)
      return ctx_fail(ctx, ORAC_ERR_PARAM, "grppt of group %d is not a contiguous ordered range", g + 1);
    prev_last = a1 + 1;
    const int n = a1 - a0 + 1;
    if (n > ORAC_MAXG)
      return ctx_fail(ctx, ORAC_ERR_PARAM, "group %d has %d atoms; at most %d are supported", g + 1, n, ORAC_MAXG);
    maxg = n > maxg ? n : maxg;
    const int ss = ss_index[a0];
    if (ss != 1 && ss != 2) return ctx_fail(ctx, ORAC_ERR_PARAM, "ss_index of atom %d is %d", a0 + 1, ss);
    gmeta[g] = make_int2(a0, n | (ss << 8));  // LJ-atom mask added below
    gmol[g] = atomp[a0] - 1;
    for (int a = a0; a <= a1; a++) {
      if (atomg[a] != g + 1) return ctx_fail(ctx, ORAC_ERR_PARAM, "atomg(%d) != %d", a + 1, g + 1);
      if (atomp[a] != atomp[a0])
        return ctx_fail(ctx, ORAC_ERR_PARAM, "group %d spans molecules %d and %d", g + 1, atomp[a0], atomp[a]);
    }
  }
  if (prev_last != N) return ctx_fail(ctx, ORAC_ERR_PARAM, "groups cover %d of %d atoms", prev_last, N);
  for (int a = 0; a < N; a++) {
    if (atomp[a] < 1 || atomp[a] > P) return ctx_fail(ctx, ORAC_ERR_PARAM, "atomp(%d) = %d", a + 1, atomp[a]);
    if (nbtype[a] < 1 || nbtype[a] > ntype) return ctx_fail(ctx, ORAC_ERR_PARAM, "nbtype(%d) = %d", a + 1, nbtype[a]);
    agrp[a] = atomg[a] - 1;
    amol[a] = atomp[a] - 1;
    atype[a] = nbtype[a] - 1;
    apm[a] = (float)pmass[a];
    aq[a] = (float)chrge[a];
    minf[a] = mass[a] >= massinfty ? 1 : 0;
  }
  // LJ table (type(ma,ma) -> ecc index), flagged off when ecc6 <= 1e-12
  const int npair = ntype * (ntype + 1) / 2;
  std::vector<float2> lj((size_t)ntype * ntype);
  std::vector<double2> ljd((size_t)ntype * ntype);
  for (int t1 = 0; t1 < ntype; t1++)
    for (int t2 = 0; t2 < ntype; t2++) {
      const int lij = type_table[t1 + (size_t)ntype * t2];
      if (lij < 1 || lij > npair) return ctx_fail(ctx, ORAC_ERR_PARAM, "type(%d,%d) = %d", t1 + 1, t2 + 1, lij);
      const double c12 = ecc12[lij - 1], c6 = ecc6[lij - 1];
      const bool on = c6 > 1e-12;  // src/force.f:416,431
      lj[t1 * (size_t)ntype + t2] = on ? make_float2((float)c12, (float)c6) : make_float2(0.f, 0.f);
      ljd[t1 * (size_t)ntype + t2] = on ? make_double2(c12, c6) : make_double2(0.0, 0.0);
      if (on && (float)c6 == 0.f)
        return ctx_fail(ctx, ORAC_ERR_PARAM, "ecc6(%d) = %g underflows single precision", lij, c6);
    }
  // atoms whose type has no LJ partner at all: under lskip_ewald every pair
  // of theirs is skipped (src/force.f:416-417), and the pair kernel skips
  // them without a table lookup; bit a of gmeta.y >> 16 marks atom a of the
  // group as having LJ
  {
    std::vector<unsigned char> tlj(ntype, 0);
    for (int t1 = 0; t1 < ntype; t1++)
      for (int t2 = 0; t2 < ntype; t2++)
        if (lj[t1 * (size_t)ntype + t2].y != 0.f) tlj[t1] = 1;
    for (int g = 0; g < G; g++) {
      int m = 0;
      for (int a = 0; a < (gmeta[g].y & 0xff); a++)
        if (tlj[nbtype[gmeta[g].x + a] - 1]) m |= 1 << a;
      gmeta[g].y |= m << 16;
    }
  }
  // exclusions: serial mapnl -> CSR with 0-based partners
  std::vector<int> exoff(N + 1), exj;
  {
    int64_t p = 0;
    for (int a = 0; a < N; a++) {
      if (p >= nmapnl) return ctx_fail(ctx, ORAC_ERR_PARAM, "mapnl ends before atom %d", a + 1);
      const int n = mapnl[p];
      if (n < 0 || p + 1 + n > nmapnl) return ctx_fail(ctx, ORAC_ERR_PARAM, "mapnl record of atom %d", a + 1);
      exoff[a] = (int)exj.size();
      for (int q = 0; q < n; q++) {
        const int j = mapnl[p + 1 + q];
        if (j <= a + 1 || j > N) return ctx_fail(ctx, ORAC_ERR_PARAM, "mapnl partner %d of atom %d", j, a + 1);
        exj.push_back(j - 1);
      }
      p += n + 1;
    }
    exoff[N] = (int)exj.size();
  }
  ctx->N = N;
  ctx->G = G;
  ctx->P = P;
  ctx->ntype = ntype;
  ctx->maxg = maxg;
  ctx->massinfty = massinfty;
  ctx->h_gfirst.resize(G);
  ctx->h_gn.resize(G);
  for (int g = 0; g < G; g++) {
    ctx->h_gfirst[g] = gmeta[g].x;
    ctx->h_gn[g] = gmeta[g].y & 0xff;
  }
  ctx->h_amol = amol;
  ctx->h_gmol = gmol;
  ctx->h_intra_b.clear();  // bonded terms of an earlier topology no longer apply
  ctx->h_intra_p.clear();
  ctx->h_charge.assign(chrge, chrge + N);
  ctx->h_mass.assign(mass, mass + N);
  ctx->h_ss.assign(ss_index, ss_index + N);
  ctx->h_nbtype.assign(nbtype, nbtype + N);
  ctx->h_ecc12.assign(ecc12, ecc12 + npair);
  ctx->h_ecc6.assign(ecc6, ecc6 + npair);
#define UP(dst, vec)                                                                                          \
  do {                                                                                                       \
    if (dev_alloc(ctx, &dst, vec.size())) return ORAC_ERR_CUDA;                                             \
    CK(cudaMemcpy(dst, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice));                   \
  } while (0)
  UP(ctx->d_gmeta, gmeta);
  UP(ctx->d_gmol, gmol);
  UP(ctx->d_agrp, agrp);
  UP(ctx->d_amol, amol);
  UP(ctx->d_atype, atype);
  UP(ctx->d_apm, apm);
  UP(ctx->d_aq, aq);
  UP(ctx->d_amassinf, minf);
  UP(ctx->d_lj, lj);
  UP(ctx->d_ljd, ljd);
  UP(ctx->d_exoff, exoff);
  if (exj.empty()) exj.push_back(0);
  UP(ctx->d_exj, exj);
  std::vector<double> qd(chrge, chrge + N);
  UP(ctx->d_aqd, qd);
#undef UP
  if (dev_alloc(ctx, &ctx->d_xyz, 3 * (size_t)N) || dev_alloc(ctx, &ctx->d_grp, 3 * (size_t)G) ||
      dev_alloc(ctx, &ctx->d_mol, 3 * (size_t)P) || dev_alloc(ctx, &ctx->d_gpos, G) ||
      dev_alloc(ctx, &ctx->d_aoff, N) || dev_alloc(ctx, &ctx->d_ffix, 3 * (size_t)N) ||
      dev_alloc(ctx, &ctx->d_fout, 3 * (size_t)N) || dev_alloc(ctx, &ctx->d_cell_of, G) ||
      dev_alloc(ctx, &ctx->d_cell_grp, G))
    return ORAC_ERR_CUDA;
  // lists: H owns the row offsets, L and M share them
  for (int q = 0; q < 3; q++) {
    GList& L = ctx->lists[q];
    if (q == 0) {
      if (dev_alloc(ctx, &L.off, G + 1)) return ORAC_ERR_CUDA;
    }
    if (dev_alloc(ctx, &L.cnt, G)) return ORAC_ERR_CUDA;
    L.valid = false;
  }
  ctx->lists[1].off = ctx->lists[0].off;
  ctx->lists[2].off = ctx->lists[0].off;
  ctx->have_topo = true;
  return ORAC_OK;
}

int orac_gpu_set_ewald(orac_gpu_ctx* ctx, int clewld, double alphal, int order, int nfft1, int nfft2, int nfft3,
                       double rkcut) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx) return ORAC_ERR_PARAM;
  if (clewld && (alphal <= 0 || order < 3 || order > 12 || nfft1 < order || nfft2 < order || nfft3 < order ||
                 nfft1 > 512 || nfft2 > 512 || nfft3 > 512))
    return ctx_fail(ctx, ORAC_ERR_PARAM, "bad PME parameters alpha=%g order=%d grid=%dx%dx%d", alphal, order, nfft1,
                    nfft2, nfft3);
  bump.arm();
  ctx->clewld = clewld ? 1 : 0;
  ctx->alphal = alphal;
  ctx->order = order;
  ctx->nfft1 = nfft1;
  ctx->nfft2 = nfft2;
  ctx->nfft3 = nfft3;
  ctx->rkcut = rkcut;
  ctx->have_ewald = true;
  if (clewld) return pme_setup(ctx, nfft1, nfft2, nfft3, order);
  return ORAC_OK;
}

int orac_gpu_set_shells(orac_gpu_ctx* ctx, double rcutm, double rtolm, double rneim, double rcutl, double rtoll,
                        double rneil, double rcuth, double rtolh, double rneih) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx) return ORAC_ERR_PARAM;
  bump.arm();
  ctx->sh = {rcutm, rtolm, rneim, rcutl, rtoll, rneil, rcuth, rtolh, rneih};
  ctx->have_shells = true;
  return ORAC_OK;
}

int orac_gpu_set_linked_cell(orac_gpu_ctx* ctx, int ncx, int ncy, int ncz) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx) return ORAC_ERR_PARAM;
  if (ncx < 0 || ncy < 0 || ncz < 0 || (long)ncx * ncy * ncz > 16 * 1024 * 1024)
    return ctx_fail(ctx, ORAC_ERR_PARAM, "bad linked cell grid");
  bump.arm();
  ctx->ncx = ncx;
  ctx->ncy = ncy;
  ctx->ncz = ncz;
  return ORAC_OK;
}

int orac_gpu_set_box(orac_gpu_ctx* ctx, const double* co, const double* oc) {
  ParamGenBump bump(ctx);  // kernels capture these values: step graphs are re-captured
  if (!ctx || !co || !oc) return ORAC_ERR_PARAM;
  if (co[1] != 0.0 || co[2] != 0.0 || co[5] != 0.0)
    return ctx_fail(ctx, ORAC_ERR_PARAM, "co must be upper triangular (ORAC's convention)");
  bump.arm();
  memcpy(ctx->co, co, sizeof(ctx->co));
  memcpy(ctx->oc, oc, sizeof(ctx->oc));
  ctx->volume = 8.0 * std::fabs(co[0] * co[4] * co[8]);
  ctx->have_box = true;
  return ORAC_OK;
}

int orac_gpu_lc_list(orac_gpu_ctx* ctx, double rcut, const double* xpga, const double* ypga, const double* zpga,
                     int64_t* npairs) {
  if (int rc = check_ready(ctx)) return rc;
  if (ctx->ncx <= 0) return ctx_fail(ctx, ORAC_ERR_STATE, "linked cells not set");
  CK(cudaSetDevice(ctx->device));
  if (int rc = upload3(ctx, ctx->d_grp, ctx->G, xpga, ypga, zpga)) return rc;
  if (int rc = list_build_cells(ctx, rcut, &ctx->lists[0])) return rc;
  if (npairs) *npairs = ctx->lists[0].npairs;
  CK(cudaStreamSynchronize(ctx->stream));
  return ORAC_OK;
}

int orac_gpu_mts_forces(orac_gpu_ctx* ctx, int nstep, char rshell, const double* xp0, const double* yp0,
                        const double* zp0, const double* xpg, const double* ypg, const double* zpg,
                        const double* xpcm, const double* ypcm, const double* zpcm, double* ucns, double* ucos,
                        double* virs, double* virsp, double* ucnp, double* ucop, double* ucnsp, double* ucosp,
                        double* fpx, double* fpy, double* fpz, double* stress) {
  (void)nstep;
  if (int rc = check_ready(ctx)) return rc;
  CK(cudaSetDevice(ctx->device));
  const int N = ctx->N;
  if (int rc = upload3(ctx, ctx->d_xyz, N, xp0, yp0, zp0)) return rc;
  if (int rc = upload3(ctx, ctx->d_grp, ctx->G, xpg, ypg, zpg)) return rc;
  if (int rc = upload3(ctx, ctx->d_mol, ctx->P, xpcm, ypcm, zpcm)) return rc;
  CK(cudaMemsetAsync(ctx->d_fout, 0, sizeof(double) * 3 * (size_t)N, ctx->stream));
  double* d_out = ctx->d_red;  // [8] energies + [9] stress
  if (int rc = shell_run(ctx, rshell, ctx->d_xyz, ctx->d_grp, ctx->d_mol, ctx->d_fout, d_out, d_out + 8, 1))
    return rc;
  if (int rc = ensure_stage(ctx, sizeof(double) * (3 * (size_t)N + 17))) return rc;
  CK(cudaMemcpyAsync(ctx->h_stage, ctx->d_fout, sizeof(double) * 3 * (size_t)N, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_stage + 3 * (size_t)N, d_out, sizeof(double) * 17, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double* f = ctx->h_stage;
  for (int a = 0; a < N; a++) {
    fpx[a] += f[a];
    fpy[a] += f[N + a];
    fpz[a] += f[2 * N + a];
  }
  const double* e = f + 3 * (size_t)N;
  *ucns = e[0];
  *ucos = e[1];
  *virs = e[2];
  *virsp = e[3];
  *ucnp = e[4];
  *ucop = e[5];
  *ucnsp = e[6];
  *ucosp = e[7];
  memcpy(stress, e + 8, 9 * sizeof(double));
  return ORAC_OK;
}

int orac_gpu_mts_forces_dev(orac_gpu_ctx* ctx, char rshell, const double* xyz_scaled, const double* grp_scaled,
                            const double* mol_scaled, double* fdev, double* energies, double* stress) {
  if (int rc = check_ready(ctx)) return rc;
  CK(cudaSetDevice(ctx->device));
  return shell_run(ctx, rshell, xyz_scaled, grp_scaled, mol_scaled, fdev, energies, stress, energies != nullptr);
}

int orac_gpu_sync(orac_gpu_ctx* ctx) {
  if (!ctx) return ORAC_ERR_PARAM;
  CK(cudaStreamSynchronize(ctx->stream));
  return ORAC_OK;
}

void* orac_gpu_get_stream(orac_gpu_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int orac_gpu_counters(orac_gpu_ctx* ctx, int64_t* out4, int reset) {
  if (!ctx) return ORAC_ERR_PARAM;
  unsigned long long h[4];
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(h, ctx->d_wcnt, sizeof(h), cudaMemcpyDeviceToHost));
  for (int k = 0; k < 4; k++) out4[k] = (int64_t)h[k];
  if (reset) CK(cudaMemset(ctx->d_wcnt, 0, sizeof(h)));
  return ORAC_OK;
}

int orac_gpu_prof_enable(orac_gpu_ctx* ctx, int on) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (on < 0 || on >= (1 << PROF_NFAM)) return ctx_fail(ctx, ORAC_ERR_PARAM, "profile mask %d", on);
  if (on && ctx->prof_ev.empty()) {
    ctx->prof_ev.resize(4096);
    ctx->prof_fam.assign(ctx->prof_ev.size() / 2, 0);
    for (auto& e : ctx->prof_ev) CK(cudaEventCreate(&e));
  }
  // the event records are nodes of the captured step graphs: a new mask
  // captures them again
  if (on != ctx->prof) ctx->param_gen++;
  ctx->prof = on;
  return ORAC_OK;
}

int orac_gpu_prof_read_family(orac_gpu_ctx* ctx, int family, double* ms_total, int64_t* nlaunch, int reset) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (family < 0 || family >= PROF_NFAM) return ctx_fail(ctx, ORAC_ERR_PARAM, "profile family %d", family);
  if (ms_total) *ms_total = ctx->prof_ms[family];
  if (nlaunch) *nlaunch = ctx->prof_bad ? -1 : ctx->prof_n[family];  // -1: some launches could not be timed
  if (reset) {
    for (int f = 0; f < PROF_NFAM; f++) {
      ctx->prof_ms[f] = 0;
      ctx->prof_n[f] = 0;
    }
    ctx->prof_bad = false;
  }
  return ORAC_OK;
}

int orac_gpu_prof_read(orac_gpu_ctx* ctx, double* ms_total, int64_t* nlaunch, int reset) {
  return orac_gpu_prof_read_family(ctx, PROF_PAIR, ms_total, nlaunch, reset);
}

int orac_gpu_stats(orac_gpu_ctx* ctx, int64_t* list_pairs, int64_t* launches) {
  if (!ctx) return ORAC_ERR_PARAM;
  if (list_pairs) {
    for (int q = 0; q < 3; q++) {
      GList& L = ctx->lists[q];
      int64_t tot = 0;
      if (L.valid && ctx->G > 0) {
        std::vector<int> c(ctx->G);
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(c.data(), L.cnt, sizeof(int) * ctx->G, cudaMemcpyDeviceToHost));
        for (int v : c) tot += v;
      }
      list_pairs[q] = tot;
    }
  }
  if (launches) *launches = ctx->launches;
  return ORAC_OK;
}

}  // extern "C"
