/*
 * ORACLE — test infrastructure only.
 *
 * FP64 CPU restatement of the r-RESPA step loop of ORAC's mtsmd
 * (src/mtsmd.f:2390-3540), NVE or with ORAC's Nose-Hoover thermostats at
 * the M level (NVT), over the restated force routines of
 * orac_oracle.c: kicks as correc (src/correc.f), drift as verlet
 * (src/verlet.f), SHAKE/RATTLE as the iterative branches of
 * src/rattle_verlet.f and src/rattle_correc.f (tolerance 1e-8 A^2,
 * 5000-iteration cap), the list update of src/mtsmd.f:2403-2470 and the
 * phony M-list refresh of :3287-3295.  It serves as the checker of the GPU
 * driver and as the timed CPU baseline (OpenMP over groups, as ORAC).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "orac_oracle.h"

static const double PI_MD = 3.14159265358979323846; /* setuns.f:35 4*atan(1) */

typedef struct {
  int ntap, ngrp, nprot, ma;
  const int *ss, *nbtype, *type, *atomg, *atomp, *grppt, *mapnl;
  const double *charge, *ecc12, *ecc6, *mass, *pmass;
  double massinfty;
  double co[9], oc[9], volume;
  double alphal, rkcut;
  int order, n1, n2, n3;
  double sh[9]; /* rcutm rtolm rneim rcutl rtoll rneil rcuth rtolh rneih */
  int ncx, ncy, ncz;
  int ncnst;
  int *cnst;
  double* dss;
  int nmolc;
  int* cstart; /* constraints sorted by molecule */
  double dth;
  int lrespa, mrespa, nupdte;
  char rshk;
  int nthreads;
  double econst;
  /* state */
  double *x, *v, *xo, *fh, *fl, *fm, *s, *g, *m;
  int *lh, *ll, *lm;
  long caph, capl, capm;
  int *indxi, *indxj, *indxk, nind;
  long step;
  double e[3][6], eer, ekin;
  /* intramolecular N0/N1 terms and the reciprocal corrections of mts_furier */
  int nb, nbend, nt, nit, n14, ningrp, n13;
  int *lbnd, *lbndg, *ltor, *litr, *int14, *type14, *ingrp, *int13;
  double *r0, *kb, *bendpot, *tpota, *tpotb, *ipota, *ipotb, *ipotc, *ecc1412, *ecc146;
  double fudge;
  int n1respa, n0respa, has_n0, has_n1;
  double *fn0, *fn1;
  double e_bonded, e_tors, e_14grp, e_ferrf;
  /* Alchemy in the loop (force_alchemy in the shells, do_pmesh_alchemy and
   * ferrf_alchemy over the scaled charges, cself_alchemy, fnb14_alchemy on
   * the N1 level, ferrf_alchemy_add over listqq after every M shell) and,
   * with a schedule, the lambdas of a non-equilibrium run (alchemic,
   * src/alchemic.f; the update of src/mtsmd.f:2963-2999) with ORAC's work
   * sum (src/mtsmd.f:3042-3044). */
  int alch, ne;
  orc_variant V;
  int* ssal;
  double *rmin, *epsm;
  int intramol, ljintra;
  double gl[4], gl0[4]; /* ladd lrm laddq lrmq and ladd0 lrm0 laddq0 lrmq0 (cpropar) */
  double *lam, *lamq, *lam0, *lamq0; /* per atom: lambda, lambdaq, lambda0, lambdaq0 */
  double *qc, *q0;                   /* chrgec, chrge0 of mts_furier_alchemy */
  int nlistqq;
  int* listqq;
  int ntimes;
  double *trec, *sch[4]; /* timerec (fs); ladded laddedq lremoved lremovedq */
  double t0, rtime;
  long ninn0;
  /* dwrkm dwrkl dwrkh dwrkrc_m dwrkrc_l dwrkrc_h dwrk_al dwrk14, and the sum */
  double dw[8], wrk;
  /* ORAC's three Nose-Hoover thermostats (THERMOS: molecular centres of
   * mass, solute, solvent), coupled at the M level
   * (src/mtsmd.f:2556-2592, 3109-3170): thermostat masses, ndf kT, the
   * coordinates eta and velocities etap, the molecules' masses */
  int thermo;
  double qmass[3], ndfkt[3], eta[3], etap[3];
  int ndf[3];
  double* tmass;
} orc_md;

/* the charge of mts_furier_alchemy (src/mts_furier_alchemy.f:96-111) */
static double alch_charge(double q, double lq) {
  const double a = fabs(lq);
  if (a == 1.0) return 0.0;
  if (a == 0.0) return q;
  return (1.0 - a) * q;
}

static void alch_refresh(orc_md* M) {
  orc_alch_set(M->V.fact, M->gl[0], M->gl[1], M->intramol, M->ljintra, 0);
  orc_alch_set(M->V.factq, M->gl[2], M->gl[3], M->intramol, M->ljintra, 1);
  orc_alch_set(M->V.fact0, M->gl0[0], M->gl0[1], M->intramol, M->ljintra, 0);
  orc_alch_set(M->V.factq0, M->gl0[2], M->gl0[3], M->intramol, M->ljintra, 1);
  for (int a = 0; a < M->ntap; a++) {
    M->qc[a] = alch_charge(M->charge[a], M->lamq[a]);
    M->q0[a] = alch_charge(M->charge[a], M->lamq0[a]);
  }
}

/* alchemic (src/alchemic.f): the lambdas of the time slice that holds
 * rtime, linear in time; the last slice that holds it wins; before the
 * first point ladd = laddq = 1, lrm = lrmq = 0; after the last point its
 * values.  sch: ladded laddedq lremoved lremovedq (ntimes each); g = ladd
 * lrm laddq lrmq. */
void orc_alchemic(int ntimes, const double* trec, const double* ladded, const double* laddedq,
                  const double* lremoved, const double* lremovedq, double rtime, double* g) {
  g[0] = 1.0;
  g[1] = 0.0;
  g[2] = 1.0;
  g[3] = 0.0;
  int i0 = -1;
  for (int i = 0; i + 1 < ntimes; i++)
    if (rtime >= trec[i] && rtime <= trec[i + 1]) i0 = i;
  if (i0 >= 0) {
    const double ts = trec[i0 + 1] - trec[i0];
    const double va = (ladded[i0 + 1] - ladded[i0]) / ts, vr = (lremoved[i0 + 1] - lremoved[i0]) / ts;
    const double vaq = (laddedq[i0 + 1] - laddedq[i0]) / ts, vrq = (lremovedq[i0 + 1] - lremovedq[i0]) / ts;
    const double dt = rtime - trec[i0];
    g[0] = ladded[i0] + va * dt;
    g[1] = lremoved[i0] + vr * dt;
    g[2] = laddedq[i0] + vaq * dt;
    g[3] = lremovedq[i0] + vrq * dt;
  }
  if (rtime > trec[ntimes - 1]) {
    const int n = ntimes - 1;
    g[0] = ladded[n];
    g[1] = lremoved[n];
    g[2] = laddedq[n];
    g[3] = lremovedq[n];
  }
}

static void alchemic(const orc_md* M, double rtime, double* g) {
  orc_alchemic(M->ntimes, M->trec, M->sch[0], M->sch[1], M->sch[2], M->sch[3], rtime, g);
}

/* the lambda update before an M shell (src/mtsmd.f:2963-2999): the
 * previous values become lambda0, the schedule gives the new ones; the
 * per-atom lambdas of the added (removed) atoms move only while ladd or
 * laddq differ from 1 (lrm or lrmq from 0) */
static void ne_update(orc_md* M) {
  for (int k = 0; k < 4; k++) M->gl0[k] = M->gl[k];
  alchemic(M, M->rtime, M->gl);
  const int add = M->gl[0] != 1.0 || M->gl[2] != 1.0;
  const int rm = M->gl[1] != 0.0 || M->gl[3] != 0.0;
  for (int a = 0; a < M->ntap; a++) {
    if (M->ssal[a] == 2 && add) {
      M->lam0[a] = M->lam[a];
      M->lamq0[a] = M->lamq[a];
      M->lam[a] = M->gl[0];
      M->lamq[a] = M->gl[2];
    } else if (M->ssal[a] == -2 && rm) {
      M->lam0[a] = M->lam[a];
      M->lam[a] = -M->gl[1];
      M->lamq0[a] = M->lamq[a];
      M->lamq[a] = -M->gl[3];
    }
  }
  alch_refresh(M);
}

/* cself_alchemy (src/cself_alchemy.f): the solute self energy of chrgec
 * minus that of chrge0 */
static double alch_self_work(const orc_md* M) {
  double s = 0.0, s0 = 0.0;
  for (int a = 0; a < M->ntap; a++)
    if (M->ss[a] == 1) {
      s += M->qc[a] * M->qc[a];
      s0 += M->q0[a] * M->q0[a];
    }
  const double f = M->alphal / sqrt(PI_MD) * (1.0 - orc_erfc_as(M->rkcut / (2.0 * M->alphal)));
  return -s * f + s0 * f;
}

#define ORC_MD_REC 16

static void md_coords(orc_md* M) {
  int N = M->ntap;
  orc_change_frame(M->co, M->oc, -1, N, M->x, M->x + N, M->x + 2 * N, M->s, M->s + N, M->s + 2 * N);
  orc_appbou(M->s, M->s + N, M->s + 2 * N, M->g, M->g + M->ngrp, M->g + 2 * M->ngrp, M->pmass, M->ngrp, M->grppt);
  int P = M->nprot;
  double* mt = (double*)calloc(P, sizeof(double));
  for (int k = 0; k < 3 * P; k++) M->m[k] = 0.0;
  for (int a = 0; a < N; a++) {
    int p = M->atomp[a] - 1;
    mt[p] += M->mass[a];
    M->m[p] += M->mass[a] * M->s[a];
    M->m[P + p] += M->mass[a] * M->s[N + a];
    M->m[2 * P + p] += M->mass[a] * M->s[2 * N + a];
  }
  for (int p = 0; p < P; p++) {
    M->m[p] /= mt[p];
    M->m[P + p] /= mt[p];
    M->m[2 * P + p] /= mt[p];
  }
  free(mt);
}

/* one call of force with explicit radii, like mts_forces (src/mts_forces.f);
 * with alchemy force_alchemy, its dwrk into *dwrk (may be null) */
static long md_force(orc_md* M, const int* in, int* out, long capout, double rneigh, double rinn, double rout,
                     double rtolinn, double rtolout, double* f, double* ue, double* dwrk) {
  int N = M->ntap, G = M->ngrp;
  double st[9] = {0};
  double uel[6];
  double extra[5] = {0, 0, 0, 0, 0};
  int lskip = orc_decide_force(rinn, M->alphal);
  double* tmp = (double*)calloc(3 * (size_t)N, sizeof(double));
  long n = orc_force_ex(M->ss, M->s, M->s + N, M->s + 2 * N, M->g, M->g + G, M->g + 2 * G, M->charge, M->nbtype,
                        M->type, M->ma, N, M->atomg, M->m, M->m + M->nprot, M->m + 2 * M->nprot, M->atomp, M->co,
                        M->ecc12, M->ecc6, M->alphal, M->mapnl, G, M->grppt, uel, tmp, tmp + N, tmp + 2 * N, st, in,
                        out, capout, rneigh, rinn, rout, rtolinn, rtolout, M->pmass, 1, M->mass, M->massinfty, lskip,
                        1, M->nthreads, M->alch ? &M->V : NULL, M->alch ? extra : NULL);
  if (f)
    for (long k = 0; k < 3 * (long)N; k++) f[k] += tmp[k];
  if (ue) memcpy(ue, uel, sizeof(uel));
  if (dwrk) *dwrk = extra[1];
  free(tmp);
  return n;
}

static int md_lists(orc_md* M) {
  int G = M->ngrp;
  double* r = M->sh;
  double rc = r[6] + r[7] + r[8];
  for (;;) {
    long n = orc_lc_list(M->ncx, M->ncy, M->ncz, M->nind, M->indxi, M->indxj, M->indxk, rc, M->co, M->g, M->g + G,
                         M->g + 2 * G, G, M->lh, M->caph);
    if (n >= 0) break;
    M->caph *= 2;
    M->lh = (int*)realloc(M->lh, sizeof(int) * M->caph);
  }
  /* phony 'h' with rcuth=rcutl, rtolh=0: ro=rcutl ri=rcutl rto=0 rti=rtoll rni=rneil */
  if (M->capl < M->caph) {
    M->capl = M->caph;
    M->ll = (int*)realloc(M->ll, sizeof(int) * M->capl);
  }
  if (md_force(M, M->lh, M->ll, M->capl, r[5], r[3], r[3], r[4], 0.0, NULL, NULL, NULL) < 0) return -1;
  /* phony 'l' with rcutl=rcutm, rtoll=0: ro=rcutm ri=rcutm rto=0 rti=rtolm rni=rneim */
  if (M->capm < M->caph) {
    M->capm = M->caph;
    M->lm = (int*)realloc(M->lm, sizeof(int) * M->capm);
  }
  if (md_force(M, M->ll, M->lm, M->capm, r[2], r[0], r[0], r[1], 0.0, NULL, NULL, NULL) < 0) return -1;
  return 0;
}

static void md_kick(orc_md* M, const double* f, double dt);
static int md_shake(orc_md* M, double dt);
static int md_rattle(orc_md* M);

/* The erf corrections of mts_furier (src/mts_furier.f:85-141) for the
 * excluded pairs: bonds and bends with forces, the 1-4 pairs with
 * fudgec = 1 - fudge (src/mtsmd.f:474), constraints energy only. */
static double md_ferrf_q(orc_md* M, const double* q, double* f);

static void md_ferrf(orc_md* M, double* f) { M->e_ferrf = md_ferrf_q(M, M->alch ? M->qc : M->charge, f); }

/* the corrections with charges q, forces into f (null: energy only);
 * returns their energy */
static double md_ferrf_q(orc_md* M, const double* q, double* f) {
  int N = M->ntap;
  double fs[2], dummy_e = 0.0, e = 0.0;
  double* scratch = (double*)calloc(3 * (size_t)N, sizeof(double));
  if (!f) f = scratch;
  if (M->nb > 0) {
    orc_ferrf(M->ss, M->alphal, q, 1.0, M->x, M->x + N, M->x + 2 * N, 1, M->lbnd, M->nb, fs, f, f + N,
              f + 2 * N);
    e += fs[0] + fs[1];
  }
  if (M->ncnst > 0) {
    orc_ferrf(M->ss, M->alphal, q, 1.0, M->x, M->x + N, M->x + 2 * N, 0, M->cnst, M->ncnst, fs, scratch,
              scratch + N, scratch + 2 * N);
    e += fs[0] + fs[1];
  }
  if (M->n13 > 0) {
    orc_ferrf(M->ss, M->alphal, q, 1.0, M->x, M->x + N, M->x + 2 * N, 1, M->int13, M->n13, fs, f, f + N,
              f + 2 * N);
    e += fs[0] + fs[1];
  }
  if (M->n14 > 0) {
    orc_ferrf(M->ss, M->alphal, q, 1.0 - M->fudge, M->x, M->x + N, M->x + 2 * N, 1, M->int14, M->n14, fs,
              f, f + N, f + 2 * N);
    e += fs[0] + fs[1];
  }
  (void)dummy_e;
  free(scratch);
  return e;
}

/* mts_intra_n0: fpbond + fpbend + fitors (src/mts_intra_n0.f:73-100) */
static void md_intra_n0(orc_md* M) {
  int N = M->ntap;
  double ue[2];
  memset(M->fn0, 0, sizeof(double) * 3 * N);
  M->e_bonded = 0.0;
  double *fx = M->fn0, *fy = M->fn0 + N, *fz = M->fn0 + 2 * N;
  const double *x = M->x, *y = M->x + N, *z = M->x + 2 * N;
  if (M->nb > 0) {
    orc_fpbond(M->ss, M->lbnd, M->nb, x, y, z, M->r0, M->kb, ue, fx, fy, fz);
    M->e_bonded += ue[0] + ue[1];
  }
  if (M->nbend > 0) {
    orc_fpbend(M->ss, M->lbndg, M->nbend, x, y, z, M->bendpot, ue, fx, fy, fz);
    M->e_bonded += ue[0] + ue[1];
  }
  if (M->nit > 0) {
    orc_fitors(M->ss, M->litr, M->nit, x, y, z, M->ipota, M->ipotb, M->ipotc, ue, fx, fy, fz);
    M->e_bonded += ue[0] + ue[1];
  }
}

/* mts_intra_n1: fptors + fnb14 + fnbgrp (src/mts_intra_n1.f:76-118); the
 * torsion energy is added to the bonded total of the last N0 call */
static void md_intra_n1(orc_md* M) {
  int N = M->ntap;
  double ue[4];
  memset(M->fn1, 0, sizeof(double) * 3 * N);
  M->e_14grp = 0.0;
  double *fx = M->fn1, *fy = M->fn1 + N, *fz = M->fn1 + 2 * N;
  const double *x = M->x, *y = M->x + N, *z = M->x + 2 * N;
  M->e_tors = 0.0;
  if (M->nt > 0) {
    orc_fptors(M->ss, M->ltor, M->nt, x, y, z, M->tpota, M->tpotb, ue, fx, fy, fz);
    M->e_tors = ue[0] + ue[1];
  }
  if (M->n14 > 0 && M->alch) {
    /* fnb14_alchemy with Ewald (src/mts_intra_n1.f:81-85): its dwrk is
     * dwrk14 (src/mtsmd.f:2903) */
    orc_fnb14_alchemy(M->ss, x, y, z, M->charge, M->ecc1412, M->ecc146, M->alphal, M->int14, M->n14, M->type14,
                      M->fudge, 1.0, M->lam, M->lamq, M->lam0, M->lamq0, fx, fy, fz, ue, &M->dw[7]);
    M->e_14grp += ue[0] + ue[1] + ue[2] + ue[3];
  } else if (M->n14 > 0) {
    orc_fnb14(M->ss, x, y, z, M->charge, N, M->ecc1412, M->ecc146, 1, 1, M->alphal, M->int14, M->n14, M->type14,
              M->fudge, 1.0, fx, fy, fz, ue);
    M->e_14grp += ue[0] + ue[1] + ue[2] + ue[3];
  }
  if (M->ningrp > 0) {
    orc_fnbgrp(M->ss, x, y, z, M->charge, M->nbtype, M->ecc12, M->ecc6, 1, M->alphal, M->ingrp, M->ningrp, fx, fy,
               fz, ue);
    M->e_14grp += ue[0] + ue[1] + ue[2] + ue[3];
  }
}

static void md_forces(orc_md* M, char sh, double* f) {
  int N = M->ntap;
  double* r = M->sh;
  const int lv = sh == 'm' ? 0 : (sh == 'l' ? 1 : 2);
  memset(f, 0, sizeof(double) * 3 * N);
  if (sh == 'm') {
    md_force(M, M->lm, NULL, 0, 0.0, 0.0, r[0], 0.0, r[1], f, M->e[0], &M->dw[0]);
  } else if (sh == 'l') {
    md_force(M, M->ll, M->lm, M->capm, r[2], r[0], r[3], r[1], r[4], f, M->e[1], &M->dw[1]);
  } else {
    md_force(M, M->lh, M->ll, M->capl, r[5], r[3], r[6], r[4], r[7], f, M->e[2], &M->dw[2]);
  }
  if (sh == 'm' && M->alch && M->nlistqq > 0) {
    /* ferrf_alchemy_add after the M shell (src/mtsmd.f:3035-3041) */
    double fs[2];
    orc_ferrf_alchemy_add(M->ss, M->alphal, M->charge, M->lamq, M->lamq0, M->x, M->x + N, M->x + 2 * N, M->listqq,
                          M->nlistqq, M->intramol, fs, &M->dw[6], f, f + N, f + 2 * N);
  }
  /* the work of the M step, before the M level's reciprocal sum */
  if (sh == 'm' && M->ne)
    for (int k = 0; k < 8; k++) M->wrk += M->dw[k];
  if (M->rshk == sh) {
    double st[9] = {0};
    const double* q = M->alch ? M->qc : M->charge;
    orc_fft_pme(N, M->s, M->s + N, M->s + 2 * N, M->m, M->m + M->nprot, M->m + 2 * M->nprot, q, M->co, M->oc,
                M->volume, M->alphal, M->order, M->n1, M->n2, M->n3, &M->eer, f, f + N, f + 2 * N, st, M->atomp, 0,
                M->rkcut, M->nthreads);
    md_ferrf(M, f);
    if (M->ne) {
      /* mts_furier_alchemy's dwrk (src/mts_furier_alchemy.f:112-186): the
       * reciprocal sum, the erf corrections and the self term of chrgec
       * minus those of chrge0 */
      double eer0 = 0.0;
      double* scr = (double*)calloc(3 * (size_t)N, sizeof(double));
      orc_fft_pme(N, M->s, M->s + N, M->s + 2 * N, M->m, M->m + M->nprot, M->m + 2 * M->nprot, M->q0, M->co,
                  M->oc, M->volume, M->alphal, M->order, M->n1, M->n2, M->n3, &eer0, scr, scr + N, scr + 2 * N, st,
                  M->atomp, 0, M->rkcut, M->nthreads);
      free(scr);
      M->dw[3 + lv] = (M->eer - eer0) + (M->e_ferrf - md_ferrf_q(M, M->q0, NULL)) + alch_self_work(M);
    }
  }
}

static void md_refresh_m(orc_md* M) {
  double* r = M->sh;
  /* phony 'l' with rcutl = rcutm: ro=rcutm rto=rtoll ri=rcutm rti=rtolm rni=rneim */
  md_force(M, M->ll, M->lm, M->capm, r[2], r[0], r[0], r[1], r[4], NULL, NULL, NULL);
}

static void md_kick(orc_md* M, const double* f, double dt) {
  int N = M->ntap;
#pragma omp parallel for num_threads(M->nthreads) schedule(static)
  for (int k = 0; k < 3 * N; k++) M->v[k] += f[k] * 0.5 * dt / M->mass[k % N];
}

/* Matrix-inversion constraint solve of one small molecule (<= 3 constraints),
 * as ORAC's MIM branch (src/rattle_verlet.f:228-330): Newton iterations for
 * the positions (shake = 1) or one exact solve for the velocities
 * (shake = 0).  Constraint k joins atoms ca[k], cb[k] (global indices). */
static int solve_small(int n, double A[3][3], double* b) {
  for (int k = 0; k < n; k++) {
    if (A[k][k] == 0.0) return 0;
    for (int i = k + 1; i < n; i++) {
      double f = A[i][k] / A[k][k];
      for (int j = k; j < n; j++) A[i][j] -= f * A[k][j];
      b[i] -= f * b[k];
    }
  }
  for (int k = n - 1; k >= 0; k--) {
    double s = b[k];
    for (int j = k + 1; j < n; j++) s -= A[k][j] * b[j];
    b[k] = s / A[k][k];
  }
  return 1;
}

static double cfac(orc_md* M, int ak, int bk, int al, int bl) {
  double ia = 1.0 / M->mass[ak], ib = 1.0 / M->mass[bk];
  return (ak == al ? ia : 0.0) - (ak == bl ? ia : 0.0) - (bk == al ? ib : 0.0) + (bk == bl ? ib : 0.0);
}

static int mim_molecule(orc_md* M, int c0, int nc, double dt, int shake) {
  int N = M->ntap;
  int ca[3], cb[3];
  double r0[3][3], lam[3] = {0, 0, 0};
  for (int k = 0; k < nc; k++) {
    ca[k] = M->cnst[2 * (c0 + k)] - 1;
    cb[k] = M->cnst[2 * (c0 + k) + 1] - 1;
    const double* ref = shake ? M->xo : M->x;
    for (int d = 0; d < 3; d++) r0[k][d] = ref[d * N + ca[k]] - ref[d * N + cb[k]];
  }
  if (!shake) { /* exact RATTLE velocity projection */
    double A[3][3], rhs[3];
    for (int k = 0; k < nc; k++) {
      double vab = 0;
      for (int d = 0; d < 3; d++) vab += r0[k][d] * (M->v[d * N + ca[k]] - M->v[d * N + cb[k]]);
      rhs[k] = -vab;
      for (int l = 0; l < nc; l++)
        A[k][l] = cfac(M, ca[k], cb[k], ca[l], cb[l]) *
                  (r0[k][0] * r0[l][0] + r0[k][1] * r0[l][1] + r0[k][2] * r0[l][2]);
    }
    if (!solve_small(nc, A, rhs)) return 0;
    for (int l = 0; l < nc; l++)
      for (int d = 0; d < 3; d++) {
        M->v[d * N + ca[l]] += rhs[l] * r0[l][d] / M->mass[ca[l]];
        M->v[d * N + cb[l]] -= rhs[l] * r0[l][d] / M->mass[cb[l]];
      }
    return 1;
  }
  int ok = 0;
  for (int it = 0; it < 50; it++) {
    double dk[3][3], g[3], gmax = 0, J[3][3];
    for (int k = 0; k < nc; k++) {
      for (int d = 0; d < 3; d++) dk[k][d] = M->x[d * N + ca[k]] - M->x[d * N + cb[k]];
      g[k] = -(dk[k][0] * dk[k][0] + dk[k][1] * dk[k][1] + dk[k][2] * dk[k][2] - M->dss[c0 + k]);
      if (fabs(g[k]) > gmax) gmax = fabs(g[k]);
    }
    if (gmax < 1e-12) {
      ok = 1;
      break;
    }
    for (int k = 0; k < nc; k++)
      for (int l = 0; l < nc; l++)
        J[k][l] = 2.0 * cfac(M, ca[k], cb[k], ca[l], cb[l]) *
                  (dk[k][0] * r0[l][0] + dk[k][1] * r0[l][1] + dk[k][2] * r0[l][2]);
    if (!solve_small(nc, J, g)) return 0;
    for (int l = 0; l < nc; l++) {
      lam[l] += g[l];
      for (int d = 0; d < 3; d++) {
        M->x[d * N + ca[l]] += g[l] * r0[l][d] / M->mass[ca[l]];
        M->x[d * N + cb[l]] -= g[l] * r0[l][d] / M->mass[cb[l]];
      }
    }
  }
  if (dt != 0.0)
    for (int l = 0; l < nc; l++)
      for (int d = 0; d < 3; d++) {
        M->v[d * N + ca[l]] += lam[l] * r0[l][d] / M->mass[ca[l]] / dt;
        M->v[d * N + cb[l]] -= lam[l] * r0[l][d] / M->mass[cb[l]] / dt;
      }
  return ok;
}

static int md_shake(orc_md* M, double dt) {
  int N = M->ntap, fail = 0;
  double dti = dt != 0.0 ? 1.0 / dt : 0.0;
#pragma omp parallel for num_threads(M->nthreads) schedule(static) reduction(| : fail)
  for (int mo = 0; mo < M->nmolc; mo++) {
    int it;
    if (M->cstart[mo + 1] - M->cstart[mo] <= 3) {
      if (!mim_molecule(M, M->cstart[mo], M->cstart[mo + 1] - M->cstart[mo], dt, 1)) fail = 1;
      continue;
    }
    for (it = 0; it < 5000; it++) {
      int moved = 0;
      for (int k = M->cstart[mo]; k < M->cstart[mo + 1]; k++) {
        int a = M->cnst[2 * k] - 1, b = M->cnst[2 * k + 1] - 1;
        double dx = M->x[a] - M->x[b], dy = M->x[N + a] - M->x[N + b], dz = M->x[2 * N + a] - M->x[2 * N + b];
        double dcnt = dx * dx + dy * dy + dz * dz - M->dss[k];
        if (fabs(dcnt) >= 1.0e-8) {
          moved = 1;
          double rx = M->xo[a] - M->xo[b], ry = M->xo[N + a] - M->xo[N + b], rz = M->xo[2 * N + a] - M->xo[2 * N + b];
          double ia = 1.0 / M->mass[a], ib = 1.0 / M->mass[b];
          double gg = dcnt / ((dx * rx + dy * ry + dz * rz) * 2.0 * (ia + ib));
          double ga = -gg * ia, gb = gg * ib;
          M->x[a] += rx * ga;
          M->x[b] += rx * gb;
          M->x[N + a] += ry * ga;
          M->x[N + b] += ry * gb;
          M->x[2 * N + a] += rz * ga;
          M->x[2 * N + b] += rz * gb;
          M->v[a] += rx * ga * dti;
          M->v[b] += rx * gb * dti;
          M->v[N + a] += ry * ga * dti;
          M->v[N + b] += ry * gb * dti;
          M->v[2 * N + a] += rz * ga * dti;
          M->v[2 * N + b] += rz * gb * dti;
        }
      }
      if (!moved) break;
    }
    if (it == 5000) fail = 1;
  }
  return fail;
}

static int md_rattle(orc_md* M) {
  int N = M->ntap, fail = 0;
#pragma omp parallel for num_threads(M->nthreads) schedule(static) reduction(| : fail)
  for (int mo = 0; mo < M->nmolc; mo++) {
    int it;
    if (M->cstart[mo + 1] - M->cstart[mo] <= 3) {
      if (!mim_molecule(M, M->cstart[mo], M->cstart[mo + 1] - M->cstart[mo], 0.0, 0)) fail = 1;
      continue;
    }
    for (it = 0; it < 5000; it++) {
      int moved = 0;
      for (int k = M->cstart[mo]; k < M->cstart[mo + 1]; k++) {
        int a = M->cnst[2 * k] - 1, b = M->cnst[2 * k + 1] - 1;
        double rx = M->x[a] - M->x[b], ry = M->x[N + a] - M->x[N + b], rz = M->x[2 * N + a] - M->x[2 * N + b];
        double vx = M->v[a] - M->v[b], vy = M->v[N + a] - M->v[N + b], vz = M->v[2 * N + a] - M->v[2 * N + b];
        double dpp = rx * vx + ry * vy + rz * vz;
        if (fabs(dpp) > 1.0e-12) {
          moved = 1;
          double ia = 1.0 / M->mass[a], ib = 1.0 / M->mass[b];
          double g = -dpp / (M->dss[k] * (ia + ib));
          M->v[a] += g * ia * rx;
          M->v[b] -= g * ib * rx;
          M->v[N + a] += g * ia * ry;
          M->v[N + b] -= g * ib * ry;
          M->v[2 * N + a] += g * ia * rz;
          M->v[2 * N + b] -= g * ib * rz;
        }
      }
      if (!moved) break;
    }
    if (it == 5000) fail = 1;
  }
  return fail;
}

/* Nose-Hoover thermostats.  ORAC keeps the molecules' centre-of-mass
 * velocities apart from the atoms' velocities relative to them
 * (comp_fcm, src/comp_fcm.f); the oracle keeps atomic velocities and
 * splits them when a thermostat acts, which is the same state: v = V + u
 * with V the molecule's centre-of-mass velocity. */
static void thermo_com(const orc_md* M, double* vc) {
  const int N = M->ntap, P = M->nprot;
  memset(vc, 0, sizeof(double) * 3 * P);
  for (int a = 0; a < N; a++) {
    const int p = M->atomp[a] - 1;
    for (int d = 0; d < 3; d++) vc[3 * p + d] += M->mass[a] * M->v[d * N + a];
  }
  for (int p = 0; p < P; p++)
    for (int d = 0; d < 3; d++) vc[3 * p + d] /= M->tmass[p];
}

/* comp_thermos_forces (src/comp_thermos_forces.f), then correc_etap
 * (src/correc_etap.f): tto = sum M V^2 over molecules (thermostat 1) and
 * sum m u^2 over solute (2) and solvent (3) atoms; etap += dt (tto - ndf
 * kT) / Q, or 0 for a massless thermostat */
static void thermo_etap(orc_md* M, double dt) {
  const int N = M->ntap, P = M->nprot;
  double* vc = (double*)malloc(sizeof(double) * 3 * (P + 1));
  thermo_com(M, vc);
  double tto[3] = {0.0, 0.0, 0.0};
  for (int p = 0; p < P; p++)
    tto[0] += M->tmass[p] * (vc[3 * p] * vc[3 * p] + vc[3 * p + 1] * vc[3 * p + 1] + vc[3 * p + 2] * vc[3 * p + 2]);
  for (int a = 0; a < N; a++) {
    const int p = M->atomp[a] - 1;
    double u2 = 0.0;
    for (int d = 0; d < 3; d++) {
      const double u = M->v[d * N + a] - vc[3 * p + d];
      u2 += u * u;
    }
    tto[M->ss[a] == 1 ? 1 : 2] += M->mass[a] * u2;
  }
  free(vc);
  for (int k = 0; k < 3; k++) {
    if (fabs(M->qmass[k]) > 1.0e-7)
      M->etap[k] += dt * (tto[k] - M->ndfkt[k]) / M->qmass[k];
    else
      M->etap[k] = 0.0;
  }
}

/* correc_exp_scale (src/correc_exp_scale.f): centre-of-mass velocities by
 * exp(-dt etap1), solute and solvent atoms' relative velocities by
 * exp(-dt etap2), exp(-dt etap3) */
static void thermo_scale(orc_md* M, double dt) {
  const int N = M->ntap, P = M->nprot;
  double* vc = (double*)malloc(sizeof(double) * 3 * (P + 1));
  thermo_com(M, vc);
  const double sc = exp(-dt * M->etap[0]), s2 = exp(-dt * M->etap[1]), s3 = exp(-dt * M->etap[2]);
  for (int a = 0; a < N; a++) {
    const int p = M->atomp[a] - 1;
    const double sk = M->ss[a] == 1 ? s2 : s3;
    for (int d = 0; d < 3; d++) {
      const double V = vc[3 * p + d];
      M->v[d * N + a] = sk * (M->v[d * N + a] - V) + sc * V;
    }
  }
  free(vc);
}

/* comp_thermos_energy (src/comp_thermos_energy.f): sum ndf kT eta +
 * 1/2 Q etap^2, internal units */
static double thermo_energy(const orc_md* M) {
  double e = 0.0;
  for (int k = 0; k < 3; k++) e += M->ndfkt[k] * M->eta[k] + 0.5 * M->qmass[k] * M->etap[k] * M->etap[k];
  return e;
}

static int md_kick_r(orc_md* M, const double* f, double dt) {
  md_kick(M, f, dt);
  return md_rattle(M);
}

void* orc_md_create(int ntap, int ngrp, int nprot, int ma, const int* ss, const int* nbtype, const int* type,
                    const int* atomg, const int* atomp, const int* grppt, const int* mapnl, const double* charge,
                    const double* ecc12, const double* ecc6, const double* mass, const double* pmass,
                    double massinfty, const double* co, const double* oc, double alphal, int order, int n1, int n2,
                    int n3, double rkcut, const double* sh, int ncx, int ncy, int ncz, const int* cnst,
                    const double* dss, int ncnst, double dth, int lrespa, int mrespa, int nupdte, char rshk,
                    const double* x, const double* v, int nthreads, double econst) {
  orc_md* M = (orc_md*)calloc(1, sizeof(orc_md));
  M->n1respa = 1;
  M->n0respa = 1;
  M->ntap = ntap;
  M->ngrp = ngrp;
  M->nprot = nprot;
  M->ma = ma;
  M->ss = ss;
  M->nbtype = nbtype;
  M->type = type;
  M->atomg = atomg;
  M->atomp = atomp;
  M->grppt = grppt;
  M->mapnl = mapnl;
  M->charge = charge;
  M->ecc12 = ecc12;
  M->ecc6 = ecc6;
  M->mass = mass;
  M->pmass = pmass;
  M->massinfty = massinfty;
  memcpy(M->co, co, sizeof(M->co));
  memcpy(M->oc, oc, sizeof(M->oc));
  M->volume = 8.0 * fabs(co[0] * co[4] * co[8]);
  M->alphal = alphal;
  M->order = order;
  M->n1 = n1;
  M->n2 = n2;
  M->n3 = n3;
  M->rkcut = rkcut;
  memcpy(M->sh, sh, sizeof(M->sh));
  M->ncx = ncx;
  M->ncy = ncy;
  M->ncz = ncz;
  M->dth = dth;
  M->lrespa = lrespa;
  M->mrespa = mrespa;
  M->nupdte = nupdte;
  M->rshk = rshk;
  M->nthreads = nthreads;
  M->econst = econst;
  int N = ntap;
  M->x = (double*)malloc(sizeof(double) * 3 * N);
  M->v = (double*)malloc(sizeof(double) * 3 * N);
  M->xo = (double*)malloc(sizeof(double) * 3 * N);
  M->fh = (double*)calloc(3 * (size_t)N, sizeof(double));
  M->fl = (double*)calloc(3 * (size_t)N, sizeof(double));
  M->fm = (double*)calloc(3 * (size_t)N, sizeof(double));
  M->s = (double*)malloc(sizeof(double) * 3 * N);
  M->g = (double*)malloc(sizeof(double) * 3 * ngrp);
  M->m = (double*)malloc(sizeof(double) * 3 * nprot);
  memcpy(M->x, x, sizeof(double) * 3 * N);
  memcpy(M->v, v, sizeof(double) * 3 * N);
  /* constraints grouped by molecule (stable) */
  M->ncnst = ncnst;
  M->cnst = (int*)malloc(sizeof(int) * 2 * (ncnst + 1));
  M->dss = (double*)malloc(sizeof(double) * (ncnst + 1));
  M->cstart = (int*)malloc(sizeof(int) * (nprot + 2));
  int k2 = 0, nm = 0;
  M->cstart[0] = 0;
  int* order_k = (int*)malloc(sizeof(int) * (ncnst + 1));
  int* cntp = (int*)calloc(nprot + 1, sizeof(int));
  for (int k = 0; k < ncnst; k++) cntp[atomp[cnst[2 * k] - 1]]++;
  int* startp = (int*)calloc(nprot + 2, sizeof(int));
  for (int p = 1; p <= nprot; p++) startp[p + 1] = startp[p] + cntp[p];
  for (int k = 0; k < ncnst; k++) order_k[startp[atomp[cnst[2 * k] - 1]]++] = k;
  for (int p = 1, pos = 0; p <= nprot; p++) {
    if (!cntp[p]) continue;
    for (int q = 0; q < cntp[p]; q++, pos++) {
      int k = order_k[pos];
      M->cnst[2 * k2] = cnst[2 * k];
      M->cnst[2 * k2 + 1] = cnst[2 * k + 1];
      M->dss[k2] = dss[k];
      k2++;
    }
    M->cstart[++nm] = k2;
  }
  M->nmolc = nm;
  free(order_k);
  free(cntp);
  free(startp);
  int indmax = (2 * ncx) * (2 * ncy) * (2 * ncz) + 1;
  M->indxi = (int*)malloc(sizeof(int) * indmax);
  M->indxj = (int*)malloc(sizeof(int) * indmax);
  M->indxk = (int*)malloc(sizeof(int) * indmax);
  M->nind = orc_lc_index(indmax, ncx, ncy, ncz, sh[6] + sh[7] + sh[8], co, M->indxi, M->indxj, M->indxk);
  M->caph = M->capl = M->capm = 1 << 20;
  M->lh = (int*)malloc(sizeof(int) * M->caph);
  M->ll = (int*)malloc(sizeof(int) * M->capl);
  M->lm = (int*)malloc(sizeof(int) * M->capm);
  if (M->nind < 0) return NULL;
  md_coords(M);
  md_lists(M);
  md_forces(M, 'm', M->fm);
  md_forces(M, 'l', M->fl);
  md_forces(M, 'h', M->fh);
  md_refresh_m(M);
  return M;
}

static int* dup_i(const int* a, size_t n) {
  int* p = (int*)malloc(sizeof(int) * (n ? n : 1));
  if (n) memcpy(p, a, sizeof(int) * n);
  return p;
}
static double* dup_d(const double* a, size_t n) {
  double* p = (double*)malloc(sizeof(double) * (n ? n : 1));
  if (n) memcpy(p, a, sizeof(double) * n);
  return p;
}

/* Intramolecular terms and the N1/N0 sub-steps (mts_intra_n0/n1, the
 * n1respa/n0respa loops of src/mtsmd.f:2641-2930); recomputes the forces of
 * the starting configuration. */
void orc_md_set_intra(void* h, int nb, const int* lbnd, const double* r0, const double* kb, int nbend,
                      const int* lbndg, const double* bendpot, int nt, const int* ltor, const double* tpota,
                      const double* tpotb, int nit, const int* litr, const double* ipota, const double* ipotb,
                      const double* ipotc, int n14, const int* int14, const int* type14, const double* ecc1412,
                      const double* ecc146, int ntab14, double fudge, int ningrp, const int* ingrp, int n13,
                      const int* int13, int n1respa, int n0respa) {
  orc_md* M = (orc_md*)h;
  int N = M->ntap;
  M->nb = nb;
  M->lbnd = dup_i(lbnd, 2 * (size_t)nb);
  M->r0 = dup_d(r0, nb);
  M->kb = dup_d(kb, nb);
  M->nbend = nbend;
  M->lbndg = dup_i(lbndg, 3 * (size_t)nbend);
  M->bendpot = dup_d(bendpot, 7 * (size_t)nbend);
  M->nt = nt;
  M->ltor = dup_i(ltor, 4 * (size_t)nt);
  M->tpota = dup_d(tpota, nt);
  M->tpotb = dup_d(tpotb, nt);
  M->nit = nit;
  M->litr = dup_i(litr, 4 * (size_t)nit);
  M->ipota = dup_d(ipota, nit);
  M->ipotb = dup_d(ipotb, nit);
  M->ipotc = dup_d(ipotc, nit);
  M->n14 = n14;
  M->int14 = dup_i(int14, 2 * (size_t)n14);
  M->type14 = dup_i(type14, n14);
  M->ecc1412 = dup_d(ecc1412, ntab14);
  M->ecc146 = dup_d(ecc146, ntab14);
  M->fudge = fudge;
  M->ningrp = ningrp;
  M->ingrp = dup_i(ingrp, 2 * (size_t)ningrp);
  M->n13 = n13;
  M->int13 = dup_i(int13, 2 * (size_t)n13);
  M->n1respa = n1respa > 0 ? n1respa : 1;
  M->n0respa = n0respa > 0 ? n0respa : 1;
  M->has_n0 = (nb + nbend + nit) > 0;
  M->has_n1 = (nt + n14 + ningrp) > 0;
  M->fn0 = (double*)calloc(3 * (size_t)N, sizeof(double));
  M->fn1 = (double*)calloc(3 * (size_t)N, sizeof(double));
  if (M->has_n0) md_intra_n0(M);
  if (M->has_n1) md_intra_n1(M);
  double* fr = M->rshk == 'h' ? M->fh : (M->rshk == 'l' ? M->fl : M->fm);
  md_forces(M, M->rshk, fr);
}

static double md_ekin(orc_md* M) {
  int N = M->ntap;
  double e = 0;
  for (int a = 0; a < N; a++)
    e += 0.5 * M->mass[a] * (M->v[a] * M->v[a] + M->v[N + a] * M->v[N + a] + M->v[2 * N + a] * M->v[2 * N + a]);
  return e;
}

/* nsteps H steps; records as the GPU driver: 12 doubles every energy_every */
int orc_md_run(void* h, int nsteps, int energy_every, double* rec) {
  orc_md* M = (orc_md*)h;
  int N = M->ntap, fail = 0, nrec = 0;
  for (int k = 0; k < nsteps; k++) {
    if (M->step % M->nupdte == 0 && M->step > 0)
      if (md_lists(M)) return 3;
    fail |= md_kick_r(M, M->fh, M->dth);
    double tl = M->dth / M->lrespa, tm = tl / M->mrespa;
    for (int il = 0; il < M->lrespa; il++) {
      fail |= md_kick_r(M, M->fl, tl);
      for (int im = 0; im < M->mrespa; im++) {
        const double tm4 = 0.25 * tm;
        if (M->thermo) {
          thermo_etap(M, tm4);
          thermo_etap(M, tm4);
          thermo_scale(M, tm4);
        }
        fail |= md_kick_r(M, M->fm, tm);
        if (M->thermo) thermo_scale(M, tm4);
        const double tn1 = tm / M->n1respa, tn0 = tn1 / M->n0respa;
        for (int i1 = 0; i1 < M->n1respa; i1++) {
          if (M->has_n1) fail |= md_kick_r(M, M->fn1, tn1);
          for (int i0 = 0; i0 < M->n0respa; i0++) {
            /* verlet (src/verlet.f): the N0 half kick without RATTLE, then
             * the drift; rattle_verlet corrects both */
            memcpy(M->xo, M->x, sizeof(double) * 3 * N);
            const double ts2 = tn0 * tn0;
            for (int q = 0; q < 3 * N; q++) {
              const double fq = M->has_n0 ? M->fn0[q] : 0.0;
              M->x[q] = M->x[q] + tn0 * M->v[q] + fq * 0.5 * ts2 / M->mass[q % N];
              M->v[q] = M->v[q] + fq * 0.5 * tn0 / M->mass[q % N];
            }
            fail |= md_shake(M, tn0);
            fail |= md_rattle(M);
            md_coords(M);
            if (M->ne) { /* rtime = oldtime + ninn0 tn0 (src/mtsmd.f:2751) */
              M->ninn0++;
              M->rtime = M->t0 + (double)M->ninn0 * tn0;
            }
            if (M->has_n0) {
              md_intra_n0(M);
              fail |= md_kick_r(M, M->fn0, tn0);
            }
          }
          if (M->has_n1) {
            md_intra_n1(M);
            fail |= md_kick_r(M, M->fn1, tn1);
          }
        }
        if (M->thermo) /* verlet_free_eta */
          for (int q = 0; q < 3; q++) M->eta[q] += tm * M->etap[q];
        if (M->ne) ne_update(M);
        md_forces(M, 'm', M->fm);
        if (M->thermo) thermo_scale(M, tm4);
        fail |= md_kick_r(M, M->fm, tm);
        if (M->thermo) {
          thermo_scale(M, tm4);
          thermo_etap(M, tm4);
          thermo_etap(M, tm4);
        }
      }
      md_forces(M, 'l', M->fl);
      fail |= md_kick_r(M, M->fl, tl);
    }
    md_forces(M, 'h', M->fh);
    md_refresh_m(M);
    fail |= md_kick_r(M, M->fh, M->dth);
    M->step++;
    if (energy_every > 0 && (k + 1) % energy_every == 0) {
      double* r = rec + ORC_MD_REC * (size_t)nrec++;
      r[0] = (double)M->step;
      r[1] = md_ekin(M);
      for (int s = 0; s < 3; s++) {
        r[2 + 2 * s] = M->e[s][0] + M->e[s][1] + M->e[s][2];
        r[3 + 2 * s] = M->e[s][3] + M->e[s][4] + M->e[s][5];
      }
      r[8] = M->eer;
      r[9] = M->econst;
      r[12] = M->e_bonded + M->e_tors;
      r[13] = M->e_14grp;
      r[14] = M->e_ferrf;
      r[15] = M->ne ? M->wrk : 0.0;
      r[10] = r[1] + r[2] + r[3] + r[4] + r[5] + r[6] + r[7] + r[8] + r[9] + r[12] + r[13] + r[14];
      if (M->thermo) { /* the extended system's conserved energy */
        const double et = thermo_energy(M);
        r[10] += et;
        if (!M->ne && !M->alch) r[15] = et;
      }
      r[11] = fail;
    }
  }
  return fail ? 1 : 0;
}

/* Alchemy in the loop: force_alchemy (soft core, or with shifted the
 * shifted potential of force_ALCHEMY_shift), lam8 = ladd lrm laddq lrmq and
 * ladd0 lrm0 laddq0 lrmq0 (the per-atom lambdas follow: added ladd / laddq,
 * removed -lrm / -lrmq), listqq (ia, ib, facQ; 1-based) of the
 * intra-alchemical Coulomb correction. */
void orc_md_set_alchemy(void* h, const int* ss_alchemy, const double* rmin, const double* epsm, double qsoft,
                        double ljsoft, int opls, int shifted, double qshift, double ljshift, int intramol,
                        int ljintra, const double* lam8, const int* listqq, int nlistqq) {
  orc_md* M = (orc_md*)h;
  const int N = M->ntap;
  M->alch = 1;
  M->ssal = dup_i(ss_alchemy, N);
  M->rmin = dup_d(rmin, N);
  M->epsm = dup_d(epsm, N);
  memset(&M->V, 0, sizeof(M->V));
  M->V.mode = 2;
  M->V.ss_alchemy = M->ssal;
  M->V.rmin = M->rmin;
  M->V.epsm = M->epsm;
  M->V.qsoft = qsoft;
  M->V.ljsoft = ljsoft;
  M->V.opls = opls;
  M->V.shifted = shifted;
  M->V.qshift = qshift;
  M->V.ljshift = ljshift;
  M->intramol = intramol;
  M->ljintra = ljintra;
  for (int k = 0; k < 4; k++) {
    M->gl[k] = lam8[k];
    M->gl0[k] = lam8[4 + k];
  }
  M->lam = (double*)calloc(N, sizeof(double));
  M->lamq = (double*)calloc(N, sizeof(double));
  M->lam0 = (double*)calloc(N, sizeof(double));
  M->lamq0 = (double*)calloc(N, sizeof(double));
  M->qc = (double*)calloc(N, sizeof(double));
  M->q0 = (double*)calloc(N, sizeof(double));
  for (int a = 0; a < N; a++) {
    if (M->ssal[a] == 2) {
      M->lam[a] = M->gl[0];
      M->lamq[a] = M->gl[2];
      M->lam0[a] = M->gl0[0];
      M->lamq0[a] = M->gl0[2];
    } else if (M->ssal[a] == -2) {
      M->lam[a] = -M->gl[1];
      M->lamq[a] = -M->gl[3];
      M->lam0[a] = -M->gl0[1];
      M->lamq0[a] = -M->gl0[3];
    }
  }
  M->nlistqq = nlistqq;
  M->listqq = nlistqq > 0 ? dup_i(listqq, 3 * (size_t)nlistqq) : NULL;
  alch_refresh(M);
}

/* A non-equilibrium run: the lambdas follow the schedule (times in fs,
 * ntimes points) from time t0 on, set as ORAC sets them when it restarts a
 * steered run (src/mtsmd.f:722-758: lambda = lambda0 = the schedule's
 * values at t0 for the species whose values there are not 0 (the added
 * atoms start at 1, the removed ones at 0 otherwise)), the work is zeroed. */
void orc_md_set_schedule(void* h, int ntimes, const double* trec, const double* ladded, const double* laddedq,
                         const double* lremoved, const double* lremovedq, double t0) {
  orc_md* M = (orc_md*)h;
  const int N = M->ntap;
  M->ne = 1;
  M->ntimes = ntimes;
  M->trec = dup_d(trec, ntimes);
  M->sch[0] = dup_d(ladded, ntimes);
  M->sch[1] = dup_d(laddedq, ntimes);
  M->sch[2] = dup_d(lremoved, ntimes);
  M->sch[3] = dup_d(lremovedq, ntimes);
  M->t0 = t0;
  M->rtime = t0;
  M->ninn0 = 0;
  alchemic(M, t0, M->gl);
  for (int k = 0; k < 4; k++) M->gl0[k] = M->gl[k];
  const int add = M->gl[0] != 0.0 || M->gl[2] != 0.0;
  const int rm = M->gl[1] != 0.0 || M->gl[3] != 0.0;
  for (int a = 0; a < N; a++) {
    if (M->ssal[a] == 2) {
      M->lam[a] = M->lam0[a] = add ? M->gl[0] : 1.0;
      M->lamq[a] = M->lamq0[a] = add ? M->gl[2] : 1.0;
    } else if (M->ssal[a] == -2) {
      M->lam[a] = M->lam0[a] = rm ? -M->gl[1] : 0.0;
      M->lamq[a] = M->lamq0[a] = rm ? -M->gl[3] : 0.0;
    }
  }
  for (int k = 0; k < 8; k++) M->dw[k] = 0.0;
  M->wrk = 0.0;
  alch_refresh(M);
}

/* out[0] the work so far, out[1] rtime, out[2..5] ladd lrm laddq lrmq,
 * out[6..13] the latest work terms */
void orc_md_work(void* h, double* out) {
  orc_md* M = (orc_md*)h;
  out[0] = M->wrk;
  out[1] = M->rtime;
  for (int k = 0; k < 4; k++) out[2 + k] = M->gl[k];
  for (int k = 0; k < 8; k++) out[6 + k] = M->dw[k];
}

/* THERMOS (src/find_thermos.f, src/cov_thermos.f): temperature temp (K)
 * and the three thermostats' frequencies nu (cm^-1: centres of mass,
 * solute, solvent).  ndf: 3 per molecule for the centres of mass; 3 per
 * atom less 3 per molecule less the constraints for solute and solvent.
 * Q = 2 ndf k T / (2 pi c nu)^2, zero for a class without atoms or with one
 * degree of freedom; eta = etap = 0. */
void orc_md_set_thermostat(void* h, double temp, const double* nu) {
  orc_md* M = (orc_md*)h;
  const int N = M->ntap, P = M->nprot;
  const double avogad = 6.022140857e23, boltz = 1.38064852e-23;
  const double unitm = 1.0 / (avogad * 1000.0), unitl = 1.0e-10, unite = unitm * (unitl / 1.0e-15) * (unitl / 1.0e-15);
  const double c = 2.0 * PI_MD * 2.997925e10;
  free(M->tmass);
  M->tmass = (double*)calloc(P + 1, sizeof(double));
  int* cls = (int*)calloc(P + 1, sizeof(int));
  int nat[3] = {0, 0, 0}, nmol[3] = {0, 0, 0}, ncn[3] = {0, 0, 0};
  for (int a = 0; a < N; a++) {
    const int p = M->atomp[a] - 1, k = M->ss[a] == 1 ? 1 : 2;
    M->tmass[p] += M->mass[a];
    nat[k]++;
    if (!cls[p]) {
      cls[p] = k;
      nmol[k]++;
    }
  }
  for (int q = 0; q < M->ncnst; q++) ncn[M->ss[M->cnst[2 * q] - 1] == 1 ? 1 : 2]++;
  free(cls);
  M->ndf[0] = 3 * P;
  for (int k = 1; k < 3; k++) M->ndf[k] = 3 * nat[k] - 3 * nmol[k] - ncn[k];
  for (int k = 0; k < 3; k++) {
    const int exist = k == 0 || nat[k] > 0;
    const double om = nu[k] * c;
    M->qmass[k] = exist ? 2.0 * M->ndf[k] * boltz * temp / (om * om) / (unitm * unitl * unitl) : 0.0;
    if (M->ndf[k] == 1) M->qmass[k] = 0.0;
    M->ndfkt[k] = M->ndf[k] * boltz * temp / unite;
    M->eta[k] = M->etap[k] = 0.0;
  }
  M->thermo = 1;
}

/* a restart's thermostat state (src/readrs.f:247-251: gh = eta, vh = etap) */
void orc_md_set_thermostat_state(void* h, const double* eta, const double* etap) {
  orc_md* M = (orc_md*)h;
  for (int k = 0; k < 3; k++) {
    M->eta[k] = eta[k];
    M->etap[k] = etap[k];
  }
}

/* out: eta[3], etap[3], Q[3], ndf[3], the thermostats' energy */
void orc_md_thermostat(void* h, double* out) {
  orc_md* M = (orc_md*)h;
  for (int k = 0; k < 3; k++) {
    out[k] = M->eta[k];
    out[3 + k] = M->etap[k];
    out[6 + k] = M->qmass[k];
    out[9 + k] = M->ndf[k];
  }
  out[12] = thermo_energy(M);
}

void orc_md_get_state(void* h, double* x, double* v) {
  orc_md* M = (orc_md*)h;
  memcpy(x, M->x, sizeof(double) * 3 * M->ntap);
  memcpy(v, M->v, sizeof(double) * 3 * M->ntap);
}

void orc_md_destroy(void* h) {
  orc_md* M = (orc_md*)h;
  if (!M) return;
  free(M->x);
  free(M->v);
  free(M->xo);
  free(M->fh);
  free(M->fl);
  free(M->fm);
  free(M->s);
  free(M->g);
  free(M->m);
  free(M->cnst);
  free(M->dss);
  free(M->cstart);
  free(M->indxi);
  free(M->indxj);
  free(M->indxk);
  free(M->lh);
  free(M->ll);
  free(M->lm);
  free(M->tmass);
  void* extra[] = {M->lbnd, M->r0, M->kb, M->lbndg, M->bendpot, M->ltor, M->tpota, M->tpotb, M->litr, M->ipota,
                   M->ipotb, M->ipotc, M->int14, M->type14, M->ecc1412, M->ecc146, M->ingrp, M->int13, M->fn0, M->fn1};
  for (unsigned k = 0; k < sizeof(extra) / sizeof(extra[0]); k++) free(extra[k]);
  void* alch[] = {M->ssal, M->rmin, M->epsm, M->lam, M->lamq, M->lam0, M->lamq0, M->qc, M->q0, M->listqq,
                  M->trec, M->sch[0], M->sch[1], M->sch[2], M->sch[3]};
  for (unsigned k = 0; k < sizeof(alch) / sizeof(alch[0]); k++) free(alch[k]);
  free(M);
}
