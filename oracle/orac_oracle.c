/*
 * ORACLE — test infrastructure only (see orac_oracle.h for the parity status
 * and conventions).  An FP64 restatement of the ORAC routines named in each
 * function's comment; loop structure and arithmetic follow the Fortran so that
 * results agree to rounding.  OpenMP structure mirrors ORAC's: static
 * ownership of groups, thread-private force arrays reduced at the end
 * (src/force.f:189-192).
 */
#include "orac_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX2(a, b, ld) ((a) + (long)(ld) * (b))

/* Constants of A&S 7.1.26 as ORAC writes them (src/force.f:123-125). */
static const double AS_A1 = 0.2548296, AS_A2 = -0.28449674, AS_A3 = 1.4214137;
static const double AS_A4 = -1.453152, AS_A5 = 1.0614054, AS_QP = 0.3275911;
static const double PI_D = 3.14159265358979323846; /* setuns.f:35 4*atan(1) */

double orc_erfc_as(double x) {
  double qt = 1.0 / (1.0 + AS_QP * x);
  double expcst = exp(-x * x);
  return ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt *
         expcst;
}

/* decide_force, src/mts_forces.f:236-239 */
int orc_decide_force(double rinn, double alphal) {
  double erfcst = orc_erfc_as(alphal * rinn);
  return erfcst < 10.0e-4;
}

/* appbou, src/appbou.f:57-69 */
void orc_appbou(const double* xp0, const double* yp0, const double* zp0,
                double* xpg, double* ypg, double* zpg, const double* pmass,
                int ngrp, const int* grppt) {
  for (int n = 0; n < ngrp; n++) {
    double sx = 0, sy = 0, sz = 0;
    for (int m = grppt[2 * n] - 1; m <= grppt[2 * n + 1] - 1; m++) {
      sx += pmass[m] * xp0[m];
      sy += pmass[m] * yp0[m];
      sz += pmass[m] * zp0[m];
    }
    xpg[n] = sx;
    ypg[n] = sy;
    zpg[n] = sz;
  }
}

/* change_frame, src/change_frame.f:40-64 */
void orc_change_frame(const double* co, const double* oc, int way, int nato,
                      const double* xp0, const double* yp0, const double* zp0,
                      double* xp1, double* yp1, double* zp1) {
  const double* m = (way == 1) ? co : oc;
  for (int i = 0; i < nato; i++) {
    double x = xp0[i], y = yp0[i], z = zp0[i];
    xp1[i] = m[0] * x + m[3] * y + m[6] * z;
    yp1[i] = m[1] * x + m[4] * y + m[7] * z;
    zp1[i] = m[2] * x + m[5] * y + m[8] * z;
  }
}

/* dist_ijk, src/dist_ijk.f:3-141: squared minimum distance between cell
 * (0,0,0) and cell (ni,nj,nk) from corner pairs, refined along the edges in
 * ndtmax steps. */
static double dist_ijk(int ni, int nj, int nk, double dx, double dy, double dz,
                       const double* co) {
  static const int nv[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {0, 1, 1},
                               {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
  const int ndtmax = 500;
  double dmin = 1e8;
  int imin = 0, jmin = 0;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) {
      double lx = (ni + nv[j][0] - nv[i][0]) * dx;
      double ly = (nj + nv[j][1] - nv[i][1]) * dy;
      double lz = (nk + nv[j][2] - nv[i][2]) * dz;
      double mx = co[0] * lx + co[3] * ly + co[6] * lz;
      double my = co[1] * lx + co[4] * ly + co[7] * lz;
      double mz = co[2] * lx + co[5] * ly + co[8] * lz;
      double d = mx * mx + my * my + mz * mz;
      if (d < dmin) {
        dmin = d;
        imin = i;
        jmin = j;
      }
    }
  double lx = (ni + nv[jmin][0] - nv[imin][0]) * dx;
  double ly = (nj + nv[jmin][1] - nv[imin][1]) * dy;
  double lz = (nk + nv[jmin][2] - nv[imin][2]) * dz;
  double mx = co[0] * lx + co[3] * ly + co[6] * lz;
  double my = co[1] * lx + co[4] * ly + co[7] * lz;
  double mz = co[2] * lx + co[5] * ly + co[8] * lz;
  dmin = 1e8;
  /* sign(1.,0.5-nv) in single precision times dx/ndtmax (dist_ijk.f:101) */
  double steps[3] = {dx, dy, dz};
  for (int ax = 0; ax < 3; ax++) {
    double dt = ((0.5 - nv[jmin][ax]) >= 0 ? 1.0 : -1.0) * steps[ax] / ndtmax;
    for (int i = 1; i <= ndtmax; i++) {
      double dmx = i * co[0 + 3 * ax] * dt;
      double dmy = i * co[1 + 3 * ax] * dt;
      double dmz = i * co[2 + 3 * ax] * dt;
      double d = (mx + dmx) * (mx + dmx) + (my + dmy) * (my + dmy) +
                 (mz + dmz) * (mz + dmz);
      if (d < dmin) dmin = d;
    }
  }
  return dmin;
}

/* lc_index, src/lc_index.f:52-122; only the full stencil (n = 2) that
 * lc_list reads is returned. */
int orc_lc_index(int indmax, int ncx, int ncy, int ncz, double ctoff,
                 const double* co, int* indxi, int* indxj, int* indxk) {
  double sqcut = ctoff * ctoff;
  double dx = 2.0 / ncx, dy = 2.0 / ncy, dz = 2.0 / ncz;
  int imax = 0, jmax = 0, kmax = 0;
  int nind = 1;
  indxi[0] = indxj[0] = indxk[0] = 0;
  for (int i = 1 - ncx; i <= ncx - 1; i++)
    for (int j = 1 - ncy; j <= ncy - 1; j++)
      for (int k = 1 - ncz; k <= ncz - 1; k++) {
        double rmin = dist_ijk(i, j, k, dx, dy, dz, co);
        if (rmin < sqcut) {
          if (i == 0 && j == 0 && k == 0) continue; /* lc_index.f:85-86 */
          if (nind + 1 > indmax) return -1;
          indxi[nind] = i;
          indxj[nind] = j;
          indxk[nind] = k;
          nind++;
          if (imax < abs(i)) imax = abs(i);
          if (jmax < abs(j)) jmax = abs(j);
          if (kmax < abs(k)) kmax = abs(k);
        }
      }
  if (imax >= (ncx + 1) / 2 || jmax >= (ncy + 1) / 2 || kmax >= (ncz + 1) / 2)
    return -2; /* lc_index.f:106-122 stops here */
  return nind;
}

static inline double pbc_nint(double x) { return round(x); } /* DNINT */

/* cell coordinate, src/lc_list.f:94-102: floor of x/dx (int() plus the
 * sign correction), wrapped into [0, nc). */
static inline int lc_cell(double x, double d, int nc) {
  double x1 = x / d;
  int ix = (int)x1;
  double frac = x1 - (double)ix;
  int n = ix + (int)(((frac >= 0 ? 1.0 : -1.0) - 1.0) / 2.0);
  return ((n % nc) + nc) % nc;
}

/* lc_list, src/lc_list.f:76-201 */
long orc_lc_list(int ncx, int ncy, int ncz, int nind, const int* indxi,
                 const int* indxj, const int* indxk, double rcut,
                 const double* co, const double* xp, const double* yp,
                 const double* zp, int natp, int* nnlpp, long cap) {
  double sqcut = rcut * rcut;
  double dx = 2.0 / ncx, dy = 2.0 / ncy, dz = 2.0 / ncz;
  int ncell = ncx * ncy * ncz;
  int* headp = (int*)calloc(ncell, sizeof(int));
  int* chainp = (int*)malloc(sizeof(int) * (natp + 1));
  int* cpi = (int*)malloc(sizeof(int) * (natp + 1));
  int* cpj = (int*)malloc(sizeof(int) * (natp + 1));
  int* cpk = (int*)malloc(sizeof(int) * (natp + 1));
  for (int n = 1; n <= natp; n++) {
    int nx = lc_cell(xp[n - 1], dx, ncx);
    int ny = lc_cell(yp[n - 1], dy, ncy);
    int nz = lc_cell(zp[n - 1], dz, ncz);
    cpi[n] = nx;
    cpj[n] = ny;
    cpk[n] = nz;
    int numcell = nz + ncz * (ny + ncy * nx);
    chainp[n] = headp[numcell];
    headp[numcell] = n;
  }
  long nvtot = 0;
  long ret = 0;
  for (int n = 1; n <= natp; n++) {
    double x1 = xp[n - 1], y1 = yp[n - 1], z1 = zp[n - 1];
    long head = nvtot;
    if (head >= cap) {
      ret = -1;
      break;
    }
    int nv = 0;
    for (int m = 0; m < nind; m++) {
      int nx = ((cpi[n] + indxi[m]) % ncx + ncx) % ncx;
      int ny = ((cpj[n] + indxj[m]) % ncy + ncy) % ncy;
      int nz = ((cpk[n] + indxk[m]) % ncz + ncz) % ncz;
      int numcell = nz + ncz * (ny + ncy * nx);
      int l = headp[numcell];
      int nmin = (m == 0) ? n : 0;
      while (l > nmin) {
        if (l > n) {
          double x2 = x1 - xp[l - 1], y2 = y1 - yp[l - 1], z2 = z1 - zp[l - 1];
          /* pbc.h: pbc(x) = anint(0.5 x) */
          x2 -= 2.0 * pbc_nint(0.5 * x2);
          y2 -= 2.0 * pbc_nint(0.5 * y2);
          z2 -= 2.0 * pbc_nint(0.5 * z2);
          double xx = co[0] * x2 + co[3] * y2 + co[6] * z2;
          double yy = co[1] * x2 + co[4] * y2 + co[7] * z2;
          double zz = co[2] * x2 + co[5] * y2 + co[8] * z2;
          double d = xx * xx + yy * yy + zz * zz;
          if (d < sqcut) {
            nv++;
            if (head + nv >= cap) {
              ret = -1;
              goto done;
            }
            nnlpp[head + nv] = l;
          }
        }
        l = chainp[l];
      }
    }
    nnlpp[head] = nv;
    nvtot = head + nv + 1;
  }
  ret = nvtot;
done:
  free(headp);
  free(chainp);
  free(cpi);
  free(cpj);
  free(cpk);
  return ret;
}

/* ------------------------------------------------------------------ force */

typedef struct {
  double* fx;
  double* fy;
  double* fz;
  unsigned char* maplg; /* per atom: .TRUE. = not excluded */
  unsigned char* mapag; /* per group */
  double uconf[3], ucoul[3];
  double st[9];
  /* per-group scratch (ngrpmax) */
  int* index0;
  double *xmap0, *ymap0, *zmap0;
  int* index1;
  double *xmap1, *ymap1, *zmap1, *xmap2, *ymap2, *zmap2, *cmap2, *swrs, *dswrs;
  double *xmap3, *ymap3, *zmap3;
  int* nlist_out; /* next-shell candidates of the current group */
  double* drs;    /* alchemy: squared centre distance of each mapped group */
  double seg_ene; /* REM: energy of the selected pairs */
  double uconf0[3], ucoul0[3]; /* alchemy: energies at lambda0 */
} force_ws;

typedef struct {
  const int* ss_index;
  const double *xp0, *yp0, *zp0, *xpg, *ypg, *zpg, *charge;
  const int *nbtype, *type;
  int ma, nato;
  const int* atomg;
  const double *xpcm, *ypcm, *zpcm;
  const int* atomp;
  const double* co;
  const double *ecc12, *ecc6;
  double alphal;
  const int* mapnl;
  const long* mapoff; /* per atom offset of its mapnl record */
  const int* grppt;
  const double *gmass, *mass;
  double massinfty;
  int lskip_ewald, ewald, iz;
  double r2inn, r2out, rinn, rinn0, r2inn0, rout0, r2out0, r2neigh;
  double arsout1, arsout2, arsinn1, arsinn2, twrtpi;
  const orc_variant* V; /* NULL: standard force */
} force_args;

/* seg_select, src/rem.f90:631-645 (0-based atoms) */
static inline int seg_select(const orc_variant* V, int a, int b) {
  const int ra = V->rematom[a] != 0, rb = V->rematom[b] != 0;
  if (V->rem_kind == 0) return ra || rb;
  if (V->rem_kind == 1) return ra && rb;
  return ra != rb;
}

/* Pair loop body shared by the four loops of src/force.f:396-731.  sw < 0
 * marks the non-switched band (qforce unscaled, energies to ucoula/uconfa);
 * otherwise the switched band with weight sw and the V sum into *cmap. */
static inline void pair_eval(const force_args* A, force_ws* W, int i1, int j,
                             double xg, double yg, double zg, double xxcm,
                             double yycm, double zzcm, double chrgei, int nbti,
                             int typeij, double sw, double* uconfa,
                             double* ucoula, double* cmap) {
  const double* co = A->co;
  int lij = A->type[IDX2(nbti - 1, A->nbtype[j] - 1, A->ma)];
  double e6 = A->ecc6[lij - 1], e12 = A->ecc12[lij - 1];
  if (A->lskip_ewald && e6 < 1e-12 && A->ewald) return; /* force.f:416-417 */
  double xc = co[0] * xg + co[3] * yg + co[6] * zg;
  double yc = co[4] * yg + co[7] * zg;
  double zc = co[8] * zg;
  double rsq = xc * xc + yc * yc + zc * zc;
  double rsqi = 1.0 / rsq;
  double qforce = 0.0;
  double wsc = (sw < 0) ? 1.0 : sw;
  /* force_rem: selected pairs scale their force and S'V share */
  const int sel = A->V && A->V->mode == 1 && seg_select(A->V, i1, j);
  const double rf = sel ? A->V->rem_factor : 1.0;
  double conf = 0.0, coul = 0.0;
  if (e6 > 1e-12) {
    double r6 = rsqi * rsqi * rsqi;
    double r12 = r6 * r6;
    double ssvir = 12.0 * e12 * r12 - 6.0 * e6 * r6;
    qforce = ssvir * rsqi * wsc;
    conf = e12 * r12 - e6 * r6;
    if (sw < 0) {
      *uconfa += conf;
    } else {
      *cmap += sel ? conf * rf : conf;
      W->uconf[typeij - 1] += sw * conf;
    }
  }
  if (!A->lskip_ewald) {
    double rsp = sqrt(rsq);
    double rspqi = rsqi / rsp;
    double alphar = A->alphal * rsp;
    double qt = 1.0 / (1.0 + AS_QP * alphar);
    double expcst = exp(-alphar * alphar);
    double erfcst =
        ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) *
        qt * expcst;
    double furpar = chrgei * A->charge[j];
    coul = furpar * erfcst / rsp;
    if (sw < 0) {
      *ucoula += furpar * erfcst / rsp;
    } else {
      W->ucoul[typeij - 1] += sw * furpar * erfcst / rsp;
      *cmap += sel ? coul * rf : furpar * erfcst / rsp;
    }
    qforce += furpar * (erfcst + A->twrtpi * alphar * expcst) * rspqi * wsc;
  } else if (!A->ewald) {
    double rsp = sqrt(rsq);
    double ssvir = chrgei * A->charge[j] / rsp;
    coul = ssvir;
    if (sw < 0) {
      W->ucoul[typeij - 1] += ssvir;
    } else {
      *cmap += sel ? ssvir * rf : ssvir;
      W->ucoul[typeij - 1] += ssvir * sw;
    }
    qforce += ssvir * rsqi * wsc;
  }
  if (sel) { /* src/force_REM.f:491-495,634-678 */
    W->seg_ene += (sw < 0) ? conf + coul : sw * conf + sw * coul;
    qforce *= rf;
  }
  W->fx[i1] += qforce * xc;
  W->fy[i1] += qforce * yc;
  W->fz[i1] += qforce * zc;
  W->fx[j] -= qforce * xc;
  W->fy[j] -= qforce * yc;
  W->fz[j] -= qforce * zc;
  double qfx = qforce * xc, qfy = qforce * yc, qfz = qforce * zc;
  W->st[0] += qfx * xxcm;
  W->st[1] += qfx * yycm;
  W->st[2] += qfx * zzcm;
  W->st[3] += qfy * xxcm;
  W->st[4] += qfy * yycm;
  W->st[5] += qfy * zzcm;
  W->st[6] += qfz * xxcm;
  W->st[7] += qfz * yycm;
  W->st[8] += qfz * zzcm;
}

/* One pass of the outer group loop of src/force.f:235-838 for group i
 * (0-based), list entries lst[0..m-1] (1-based groups), first entry mbeg. */
static int force_group(const force_args* A, force_ws* W, int i, const int* lst,
                       int m, int mbeg) {
  const double* co = A->co;
  double xpgi = A->xpg[i], ypgi = A->ypg[i], zpgi = A->zpg[i];
  int map = 0, mp0 = 0, mp1 = 0;
  int typei = A->ss_index[A->grppt[2 * i] - 1];
  for (int jj = mbeg; jj < m; jj++) {
    int j = lst[jj] - 1;
    double xgg = xpgi - A->xpg[j], ygg = ypgi - A->ypg[j], zgg = zpgi - A->zpg[j];
    double xm = 2.0 * round(0.5 * xgg), ym = 2.0 * round(0.5 * ygg),
           zm = 2.0 * round(0.5 * zgg);
    xgg -= xm;
    ygg -= ym;
    zgg -= zm;
    double xc = co[0] * xgg + co[3] * ygg + co[6] * zgg;
    double yc = co[4] * ygg + co[7] * zgg;
    double zc = co[8] * zgg;
    double drj = xc * xc + yc * yc + zc * zc;
    if (A->r2inn > 1.0e-5 && drj < A->r2neigh) W->nlist_out[map++] = j + 1;
    if (A->rinn0 > sqrt(A->r2out) || A->iz == 0) continue;
    if (drj >= A->r2inn0 && drj < A->r2out) {
      W->xmap0[mp0] = xm;
      W->ymap0[mp0] = ym;
      W->zmap0[mp0] = zm;
      W->index0[mp0] = j;
      mp0++;
    } else if (drj >= A->r2out && drj < A->r2out0) {
      double rsp = sqrt(drj);
      double auxa = (A->arsout1 + 2.0 * rsp) / A->arsout2;
      double auxb = sqrt(A->r2out0) - rsp;
      W->xmap1[mp1] = xm;
      W->ymap1[mp1] = ym;
      W->zmap1[mp1] = zm;
      W->xmap2[mp1] = xc;
      W->ymap2[mp1] = yc;
      W->zmap2[mp1] = zc;
      W->index1[mp1] = j;
      W->swrs[mp1] = auxa * auxb * auxb;
      W->dswrs[mp1] = (-2.0 * auxa * auxb + 2.0 * auxb * auxb / A->arsout2) / rsp;
      mp1++;
    } else if (drj >= A->r2inn && drj < A->r2inn0) {
      double rsp = sqrt(drj);
      double auxa = (A->arsinn1 + 2.0 * rsp) / A->arsinn2;
      double auxb = A->rinn0 - rsp;
      W->xmap1[mp1] = xm;
      W->ymap1[mp1] = ym;
      W->zmap1[mp1] = zm;
      W->xmap2[mp1] = xc;
      W->ymap2[mp1] = yc;
      W->zmap2[mp1] = zc;
      W->index1[mp1] = j;
      W->swrs[mp1] = 1.0 - auxa * auxb * auxb;
      W->dswrs[mp1] = (2.0 * auxa * auxb - 2.0 * auxb * auxb / A->arsinn2) / rsp;
      mp1++;
    }
  }
  int mapa = mp0, mapb = mp1;
  for (int jj = 0; jj < mapb; jj++) W->cmap2[jj] = 0.0;
  if (mapa == 0 && mapb == 0) return map;
  int g0 = A->grppt[2 * i] - 1, g1 = A->grppt[2 * i + 1] - 1;
  for (int i1 = g0; i1 <= g1; i1++) {
    double xpi = A->xp0[i1], ypi = A->yp0[i1], zpi = A->zp0[i1];
    int nbti = A->nbtype[i1];
    double chrgei = A->charge[i1];
    const int* rec = A->mapnl + A->mapoff[i1];
    int la = rec[0];
    for (int q = 1; q <= la; q++) {
      int mm = rec[q] - 1;
      W->maplg[mm] = 0;
      W->mapag[A->atomg[mm] - 1] = 0;
    }
    int p1 = A->atomp[i1] - 1;
    double xpcmp1 = A->xpcm[p1], ypcmp1 = A->ypcm[p1], zpcmp1 = A->zpcm[p1];
    /* non-switched band, force.f:396-565 */
    for (int jj = 0; jj < mapa; jj++) {
      int j1 = W->index0[jj];
      int typej = A->ss_index[A->grppt[2 * j1] - 1];
      int typeij = typei + typej - 1;
      double xd = -W->xmap0[jj], yd = -W->ymap0[jj], zd = -W->zmap0[jj];
      double xd1 = xpi + xd, yd1 = ypi + yd, zd1 = zpi + zd;
      xd += xpcmp1;
      yd += ypcmp1;
      zd += zpcmp1;
      double uconfa = 0.0, ucoula = 0.0;
      int fast = W->mapag[j1];
      for (int j = A->grppt[2 * j1] - 1; j <= A->grppt[2 * j1 + 1] - 1; j++) {
        if (!fast) {
          if (!(W->maplg[j] &&
                (A->mass[j] < A->massinfty || A->mass[i1] < A->massinfty)))
            continue;
        }
        int p2 = A->atomp[j] - 1;
        pair_eval(A, W, i1, j, xd1 - A->xp0[j], yd1 - A->yp0[j],
                  zd1 - A->zp0[j], xd - A->xpcm[p2], yd - A->ypcm[p2],
                  zd - A->zpcm[p2], chrgei, nbti, typeij, -1.0, &uconfa,
                  &ucoula, NULL);
      }
      W->ucoul[typeij - 1] += ucoula;
      W->uconf[typeij - 1] += uconfa;
    }
    /* switched bands, force.f:569-731 */
    for (int jj = 0; jj < mapb; jj++) {
      int j1 = W->index1[jj];
      int typej = A->ss_index[A->grppt[2 * j1] - 1];
      int typeij = typei + typej - 1;
      int fast = W->mapag[j1];
      for (int j = A->grppt[2 * j1] - 1; j <= A->grppt[2 * j1 + 1] - 1; j++) {
        if (!fast) {
          if (!(W->maplg[j] &&
                (A->mass[j] < A->massinfty || A->mass[i1] < A->massinfty)))
            continue;
        }
        int p2 = A->atomp[j] - 1;
        pair_eval(A, W, i1, j, xpi - A->xp0[j] - W->xmap1[jj],
                  ypi - A->yp0[j] - W->ymap1[jj], zpi - A->zp0[j] - W->zmap1[jj],
                  xpcmp1 - A->xpcm[p2] - W->xmap1[jj],
                  ypcmp1 - A->ypcm[p2] - W->ymap1[jj],
                  zpcmp1 - A->zpcm[p2] - W->zmap1[jj], chrgei, nbti, typeij,
                  W->swrs[jj], NULL, NULL, &W->cmap2[jj]);
      }
    }
    for (int q = 1; q <= la; q++) {
      int mm = rec[q] - 1;
      W->maplg[mm] = 1;
      W->mapag[A->atomg[mm] - 1] = 1;
    }
  }
  /* S'*V term, force.f:754-817 */
  for (int jj = 0; jj < mapb; jj++) {
    W->xmap3[jj] = -W->dswrs[jj] * W->cmap2[jj] * W->xmap2[jj];
    W->ymap3[jj] = -W->dswrs[jj] * W->cmap2[jj] * W->ymap2[jj];
    W->zmap3[jj] = -W->dswrs[jj] * W->cmap2[jj] * W->zmap2[jj];
  }
  if (mapb != 0) {
    for (int i1 = g0; i1 <= g1; i1++) {
      double massi = A->gmass[i1];
      int p1 = A->atomp[i1] - 1;
      double xp1 = A->xpcm[p1], yp1 = A->ypcm[p1], zp1 = A->zpcm[p1];
      for (int jj = 0; jj < mapb; jj++) {
        W->fx[i1] += massi * W->xmap3[jj];
        W->fy[i1] += massi * W->ymap3[jj];
        W->fz[i1] += massi * W->zmap3[jj];
        W->st[0] += massi * W->xmap3[jj] * xp1;
        W->st[1] += massi * W->xmap3[jj] * yp1;
        W->st[2] += massi * W->xmap3[jj] * zp1;
        W->st[3] += massi * W->ymap3[jj] * xp1;
        W->st[4] += massi * W->ymap3[jj] * yp1;
        W->st[5] += massi * W->ymap3[jj] * zp1;
        W->st[6] += massi * W->zmap3[jj] * xp1;
        W->st[7] += massi * W->zmap3[jj] * yp1;
        W->st[8] += massi * W->zmap3[jj] * zp1;
      }
    }
    for (int jj = 0; jj < mapb; jj++) {
      int j = W->index1[jj];
      double xxcm = W->xmap1[jj], yycm = W->ymap1[jj], zzcm = W->zmap1[jj];
      for (int j1 = A->grppt[2 * j] - 1; j1 <= A->grppt[2 * j + 1] - 1; j1++) {
        double massj = A->gmass[j1];
        W->fx[j1] -= massj * W->xmap3[jj];
        W->fy[j1] -= massj * W->ymap3[jj];
        W->fz[j1] -= massj * W->zmap3[jj];
        int p2 = A->atomp[j1] - 1;
        double xq = -(A->xpcm[p2] + xxcm) * massj;
        double yq = -(A->ypcm[p2] + yycm) * massj;
        double zq = -(A->zpcm[p2] + zzcm) * massj;
        W->st[0] += W->xmap3[jj] * xq;
        W->st[1] += W->xmap3[jj] * yq;
        W->st[2] += W->xmap3[jj] * zq;
        W->st[3] += W->ymap3[jj] * xq;
        W->st[4] += W->ymap3[jj] * yq;
        W->st[5] += W->ymap3[jj] * zq;
        W->st[6] += W->zmap3[jj] * xq;
        W->st[7] += W->zmap3[jj] * yq;
        W->st[8] += W->zmap3[jj] * zq;
      }
    }
  }
  return map;
}

/* Shifted-potential pair of force_ALCHEMY_shift,
 * src/force_alchemy_shifted.f:466-520: the LJ distance r + ljshift sigma
 * two6 alch_fact(1,t) (two6 = 2**(1./6.) with a single-precision
 * exponent, :178), the Coulomb denominator r + qshift alch_factq(1,t), the
 * erfc taken at the unshifted r. */
static void alch_pair_shift(const force_args* A, force_ws* W, int i1, int j, int j1, double xc, double yc,
                            double zc, double xxcm, double yycm, double zzcm, double rsq, double sigma,
                            double epsmin, double chrgei, int typeij, int t, double sw) {
  const orc_variant* V = A->V;
  const double two6 = pow(2.0, (double)(1.0f / 6.0f));
  double r = sqrt(rsq);
  double qforce;
  if (epsmin > 1.0e-12) {
    double rl = r + V->ljshift * sigma * two6 * V->fact[0][t];
    double rl0 = r + V->ljshift * sigma * two6 * V->fact0[0][t];
    double r6 = pow(sigma / rl, 6.0);
    double r60 = pow(sigma / rl0, 6.0);
    double ssvirr = V->fact[1][t] * epsmin * (12.0 * r6 * r6 - 6.0 * r6);
    double ucon = V->fact[1][t] * epsmin * (r6 * r6 - r6);
    double ucon0 = V->fact0[1][t] * epsmin * (r60 * r60 - r60);
    qforce = ssvirr * sw / (r * rl);
    W->cmap2[j1] += ucon;
    W->uconf[typeij - 1] += sw * ucon;
    W->uconf0[typeij - 1] += sw * ucon0;
  } else {
    qforce = 0.0;
  }
  double rq = r + V->qshift * V->factq[0][t];
  double rq0 = r + V->qshift * V->factq0[0][t];
  if (!A->lskip_ewald) {
    double alphar = A->alphal * r;
    double qt = 1.0 / (1.0 + AS_QP * alphar);
    double expcst = exp(-alphar * alphar);
    double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
    double furpar = V->factq[1][t] * chrgei * A->charge[j];
    double furpar0 = V->factq0[1][t] * chrgei * A->charge[j];
    W->ucoul[typeij - 1] += sw * furpar * erfcst / rq;
    W->ucoul0[typeij - 1] += sw * furpar0 * erfcst / rq0;
    W->cmap2[j1] += furpar * erfcst / rq;
    qforce += furpar * (erfcst * sw / (rq * rq * r) + A->twrtpi * alphar * expcst * sw / (r * r * rq));
  } else if (!A->ewald) {
    double ssvir = V->factq[1][t] * chrgei * A->charge[j] / rq;
    double ssvir0 = V->factq0[1][t] * chrgei * A->charge[j] / rq0;
    W->cmap2[j1] += ssvir;
    W->ucoul[typeij - 1] += ssvir * sw;
    W->ucoul0[typeij - 1] += ssvir0 * sw;
    qforce += ssvir * sw / (rq * r);
  }
  W->fx[i1] += qforce * xc;
  W->fy[i1] += qforce * yc;
  W->fz[i1] += qforce * zc;
  W->fx[j] -= qforce * xc;
  W->fy[j] -= qforce * yc;
  W->fz[j] -= qforce * zc;
  W->st[0] += qforce * xc * xxcm;
  W->st[1] += qforce * xc * yycm;
  W->st[2] += qforce * xc * zzcm;
  W->st[3] += qforce * yc * xxcm;
  W->st[4] += qforce * yc * yycm;
  W->st[5] += qforce * yc * zzcm;
  W->st[6] += qforce * zc * xxcm;
  W->st[7] += qforce * zc * yycm;
  W->st[8] += qforce * zc * zzcm;
}

/* Soft-core pair of force_alchemy, src/force_alchemy.f:441-531.  j1 is the
 * map slot of the partner group. */
static inline void alch_pair(const force_args* A, force_ws* W, int i1, int j,
                             int j1, double xpi, double ypi, double zpi,
                             double xpcmp1, double ypcmp1, double zpcmp1,
                             double chrgei, int typeij) {
  const orc_variant* V = A->V;
  const double* co = A->co;
  double sigma = V->opls ? 2.0 * sqrt(V->rmin[j] * V->rmin[i1])
                         : V->rmin[j] + V->rmin[i1];
  double epsmin = 4.0 * sqrt(V->epsm[i1] * V->epsm[j]);
  if (epsmin < 1.0e-12 && A->lskip_ewald && A->ewald) return;
  const int t = V->ss_alchemy[i1] + V->ss_alchemy[j] + 4;
  const double sw = W->swrs[j1];
  int p2 = A->atomp[j] - 1;
  double xxcm = xpcmp1 - A->xpcm[p2] - W->xmap1[j1];
  double yycm = ypcmp1 - A->ypcm[p2] - W->ymap1[j1];
  double zzcm = zpcmp1 - A->zpcm[p2] - W->zmap1[j1];
  double xg = xpi - A->xp0[j] - W->xmap1[j1];
  double yg = ypi - A->yp0[j] - W->ymap1[j1];
  double zg = zpi - A->zp0[j] - W->zmap1[j1];
  double xc = co[0] * xg + co[3] * yg + co[6] * zg;
  double yc = co[4] * yg + co[7] * zg;
  double zc = co[8] * zg;
  double rsq = xc * xc + yc * yc + zc * zc;
  double auxa = 1.0 / sqrt(rsq);
  if (V->shifted) {
    alch_pair_shift(A, W, i1, j, j1, xc, yc, zc, xxcm, yycm, zzcm, rsq, sigma, epsmin, chrgei, typeij, t, sw);
    return;
  }
  double fq = V->factq[0][t], fq0 = V->factq0[0][t];
  double auxaa = 1.0 / sqrt(V->qsoft * (fq * fq) + rsq); /* soft core */
  double auxa0 = 1.0 / sqrt(V->qsoft * (fq0 * fq0) + rsq);
  double auxbb = auxaa * auxaa * auxaa;
  double qforce;
  if (epsmin > 1.0e-12) {
    double r6 = rsq * rsq * rsq / pow(sigma, 6.0);
    double gp = V->ljsoft * V->fact[0][t] + r6;
    double gp1 = 1.0 / gp;
    double gp2 = gp1 * gp1;
    double gp0 = V->ljsoft * V->fact0[0][t] + r6;
    double gp10 = 1.0 / gp0;
    double gp20 = gp10 * gp10;
    double gr = 6.0 * r6 * auxa;
    double ssvir = V->fact[1][t] * epsmin * (2.0 * gp1 * gp2 - gp2);
    double ssvirr = gr * ssvir;
    double auxc = epsmin * (gp2 - gp1);
    double auxc0 = epsmin * (gp20 - gp10);
    double ucon = V->fact[1][t] * auxc;
    double ucon0 = V->fact0[1][t] * auxc0;
    qforce = ssvirr * sw * auxa;
    W->cmap2[j1] += ucon;
    W->uconf[typeij - 1] += sw * ucon;
    W->uconf0[typeij - 1] += sw * ucon0;
  } else {
    qforce = 0.0;
  }
  if (!A->lskip_ewald) {
    double alphar = A->alphal / auxa;
    double qt = 1.0 / (1.0 + AS_QP * alphar);
    double expcst = exp(-alphar * alphar);
    double erfcst =
        ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) *
        qt * expcst;
    double furpar = V->factq[1][t] * chrgei * A->charge[j];
    double furpar0 = V->factq0[1][t] * chrgei * A->charge[j];
    W->ucoul[typeij - 1] += sw * furpar * erfcst * auxaa;
    W->ucoul0[typeij - 1] += sw * furpar0 * erfcst * auxa0;
    W->cmap2[j1] += furpar * erfcst * auxaa;
    qforce += furpar * erfcst * auxbb * sw +
              furpar * A->twrtpi * alphar * expcst * auxa * auxa * auxaa * sw;
  } else if (!A->ewald) {
    double auxc = chrgei * A->charge[j] * auxaa;
    double ssvir = V->factq[1][t] * auxc;
    double ssvir0 = V->factq0[1][t] * chrgei * A->charge[j] * auxa0;
    W->cmap2[j1] += ssvir;
    W->ucoul[typeij - 1] += ssvir * sw;
    W->ucoul0[typeij - 1] += ssvir0 * sw;
    qforce += ssvir * sw * auxaa * auxaa;
  }
  W->fx[i1] += qforce * xc;
  W->fy[i1] += qforce * yc;
  W->fz[i1] += qforce * zc;
  W->fx[j] -= qforce * xc;
  W->fy[j] -= qforce * yc;
  W->fz[j] -= qforce * zc;
  W->st[0] += qforce * xc * xxcm;
  W->st[1] += qforce * xc * yycm;
  W->st[2] += qforce * xc * zzcm;
  W->st[3] += qforce * yc * xxcm;
  W->st[4] += qforce * yc * yycm;
  W->st[5] += qforce * yc * zzcm;
  W->st[6] += qforce * zc * xxcm;
  W->st[7] += qforce * zc * yycm;
  W->st[8] += qforce * zc * zzcm;
}

/* One group of force_alchemy's outer loop, src/force_alchemy.f:261-650:
 * every partner in [rinn, rout0) is mapped once, with S = 1 on the
 * non-switched band, and exclusions and fixed-mass pairs are always checked
 * (there is no per-group fast path). */
static int force_group_alch(const force_args* A, force_ws* W, int i,
                            const int* lst, int m, int mbeg) {
  const double* co = A->co;
  double xpgi = A->xpg[i], ypgi = A->ypg[i], zpgi = A->zpg[i];
  int map = 0, mp = 0;
  int typei = A->ss_index[A->grppt[2 * i] - 1];
  const double rout = sqrt(A->r2out);
  for (int jj = mbeg; jj < m; jj++) {
    int j = lst[jj] - 1;
    double xgg = xpgi - A->xpg[j], ygg = ypgi - A->ypg[j], zgg = zpgi - A->zpg[j];
    double xm = 2.0 * round(0.5 * xgg), ym = 2.0 * round(0.5 * ygg),
           zm = 2.0 * round(0.5 * zgg);
    xgg -= xm;
    ygg -= ym;
    zgg -= zm;
    double xc = co[0] * xgg + co[3] * ygg + co[6] * zgg;
    double yc = co[4] * ygg + co[7] * zgg;
    double zc = co[8] * zgg;
    double drj = xc * xc + yc * yc + zc * zc;
    if (A->r2inn > 1.0e-5 && drj < A->r2neigh) W->nlist_out[map++] = j + 1;
    if (A->rinn0 > rout) continue;
    if (drj >= A->r2inn && drj < A->r2out0) {
      W->xmap1[mp] = xm;
      W->ymap1[mp] = ym;
      W->zmap1[mp] = zm;
      W->xmap2[mp] = xc;
      W->ymap2[mp] = yc;
      W->zmap2[mp] = zc;
      W->drs[mp] = drj;
      W->index1[mp] = j;
      mp++;
    }
  }
  int mapb = mp;
  for (int jj = 0; jj < mapb; jj++) {
    double d = W->drs[jj];
    if (d < A->r2out && d >= A->r2inn0) {
      W->swrs[jj] = 1.0;
      W->dswrs[jj] = 0.0;
    } else if (d >= A->r2out) {
      double rsp = sqrt(d);
      double auxa = (A->arsout1 + 2.0 * rsp) / A->arsout2;
      double auxb = A->rout0 - rsp;
      W->swrs[jj] = auxa * auxb * auxb;
      W->dswrs[jj] = (-2.0 * auxa * auxb + 2.0 * auxb * auxb / A->arsout2) / rsp;
    } else {
      double rsp = sqrt(d);
      double auxa = (A->arsinn1 + 2.0 * rsp) / A->arsinn2;
      double auxb = A->rinn0 - rsp;
      W->swrs[jj] = 1.0 - auxa * auxb * auxb;
      W->dswrs[jj] = (2.0 * auxa * auxb - 2.0 * auxb * auxb / A->arsinn2) / rsp;
    }
    W->cmap2[jj] = 0.0;
  }
  if (mapb == 0) return map;
  int g0 = A->grppt[2 * i] - 1, g1 = A->grppt[2 * i + 1] - 1;
  for (int i1 = g0; i1 <= g1; i1++) {
    const int* rec = A->mapnl + A->mapoff[i1];
    int la = rec[0];
    for (int q = 1; q <= la; q++) W->maplg[rec[q] - 1] = 0;
    int p1 = A->atomp[i1] - 1;
    for (int jj = 0; jj < mapb; jj++) {
      int jg = W->index1[jj];
      int typej = A->ss_index[A->grppt[2 * jg] - 1];
      for (int j = A->grppt[2 * jg] - 1; j <= A->grppt[2 * jg + 1] - 1; j++) {
        if (!(W->maplg[j] &&
              (A->mass[j] < A->massinfty || A->mass[i1] < A->massinfty)))
          continue;
        alch_pair(A, W, i1, j, jj, A->xp0[i1], A->yp0[i1], A->zp0[i1],
                  A->xpcm[p1], A->ypcm[p1], A->zpcm[p1], A->charge[i1],
                  typei + typej - 1);
      }
    }
    for (int q = 1; q <= la; q++) W->maplg[rec[q] - 1] = 1;
  }
  /* S'*V term, src/force_alchemy.f:552-622 (same as force) */
  for (int jj = 0; jj < mapb; jj++) {
    W->xmap3[jj] = -W->dswrs[jj] * W->cmap2[jj] * W->xmap2[jj];
    W->ymap3[jj] = -W->dswrs[jj] * W->cmap2[jj] * W->ymap2[jj];
    W->zmap3[jj] = -W->dswrs[jj] * W->cmap2[jj] * W->zmap2[jj];
  }
  for (int i1 = g0; i1 <= g1; i1++) {
    double massi = A->gmass[i1];
    int p1 = A->atomp[i1] - 1;
    double xp1 = A->xpcm[p1], yp1 = A->ypcm[p1], zp1 = A->zpcm[p1];
    for (int jj = 0; jj < mapb; jj++) {
      W->fx[i1] += massi * W->xmap3[jj];
      W->fy[i1] += massi * W->ymap3[jj];
      W->fz[i1] += massi * W->zmap3[jj];
      W->st[0] += massi * W->xmap3[jj] * xp1;
      W->st[1] += massi * W->xmap3[jj] * yp1;
      W->st[2] += massi * W->xmap3[jj] * zp1;
      W->st[3] += massi * W->ymap3[jj] * xp1;
      W->st[4] += massi * W->ymap3[jj] * yp1;
      W->st[5] += massi * W->ymap3[jj] * zp1;
      W->st[6] += massi * W->zmap3[jj] * xp1;
      W->st[7] += massi * W->zmap3[jj] * yp1;
      W->st[8] += massi * W->zmap3[jj] * zp1;
    }
  }
  for (int jj = 0; jj < mapb; jj++) {
    int j = W->index1[jj];
    double xxcm = W->xmap1[jj], yycm = W->ymap1[jj], zzcm = W->zmap1[jj];
    for (int j1 = A->grppt[2 * j] - 1; j1 <= A->grppt[2 * j + 1] - 1; j1++) {
      double massj = A->gmass[j1];
      W->fx[j1] -= massj * W->xmap3[jj];
      W->fy[j1] -= massj * W->ymap3[jj];
      W->fz[j1] -= massj * W->zmap3[jj];
      int p2 = A->atomp[j1] - 1;
      double xq = -(A->xpcm[p2] + xxcm) * massj;
      double yq = -(A->ypcm[p2] + yycm) * massj;
      double zq = -(A->zpcm[p2] + zzcm) * massj;
      W->st[0] += W->xmap3[jj] * xq;
      W->st[1] += W->xmap3[jj] * yq;
      W->st[2] += W->xmap3[jj] * zq;
      W->st[3] += W->ymap3[jj] * xq;
      W->st[4] += W->ymap3[jj] * yq;
      W->st[5] += W->ymap3[jj] * zq;
      W->st[6] += W->zmap3[jj] * xq;
      W->st[7] += W->zmap3[jj] * yq;
      W->st[8] += W->zmap3[jj] * zq;
    }
  }
  return map;
}

void orc_alch_set(double fact[2][9], double ladd, double lrm, int intramol,
                  int ljintra, int qq) {
  for (int k = 0; k < 2; k++)
    for (int t = 0; t < 9; t++) fact[k][t] = 0.0;
  const double la = fabs(ladd), lr = fabs(lrm);
#define F(t, a, b) (fact[0][(t) + 4] = (a), fact[1][(t) + 4] = (b))
  F(2, 0.0, 1.0);       /* normal-normal */
  F(3, la, 1.0 - la);   /* normal-added */
  F(-1, lr, 1.0 - lr);  /* normal-removed */
  if (intramol && qq) {
    F(4, la * la, 1.0 - la * la);
    F(-4, lr * lr, 1.0 - lr * lr);
  } else if (intramol && !ljintra) {
    F(4, la, 1.0 - la);
    F(-4, lr, 1.0 - lr);
  } else {
    F(4, 0.0, 1.0);
    F(-4, 0.0, 1.0);
  }
  F(0, 0.0, 0.0); /* removed-added */
#undef F
}

long orc_force(const int* ss_index, const double* xp0, const double* yp0,
               const double* zp0, const double* xpg, const double* ypg,
               const double* zpg, const double* charge, const int* nbtype,
               const int* type, int ma, int nato, const int* atomg,
               const double* xpcm, const double* ypcm, const double* zpcm,
               const int* atomp, const double* co, const double* ecc12,
               const double* ecc6, double alphal, const int* mapnl, int ngrp,
               const int* grppt, double* ue, double* fpx, double* fpy,
               double* fpz, double* stress, const int* nnlpp, int* nnlpp1,
               long cap1, double rneigh, double rinn, double rout,
               double rtolinn, double rtolout, const double* gmass, int iz,
               const double* mass, double massinfty, int lskip_ewald,
               int ewald, int nthreads) {
  return orc_force_ex(ss_index, xp0, yp0, zp0, xpg, ypg, zpg, charge, nbtype,
                      type, ma, nato, atomg, xpcm, ypcm, zpcm, atomp, co,
                      ecc12, ecc6, alphal, mapnl, ngrp, grppt, ue, fpx, fpy,
                      fpz, stress, nnlpp, nnlpp1, cap1, rneigh, rinn, rout,
                      rtolinn, rtolout, gmass, iz, mass, massinfty,
                      lskip_ewald, ewald, nthreads, NULL, NULL);
}

long orc_force_ex(const int* ss_index, const double* xp0, const double* yp0,
                  const double* zp0, const double* xpg, const double* ypg,
                  const double* zpg, const double* charge, const int* nbtype,
                  const int* type, int ma, int nato, const int* atomg,
                  const double* xpcm, const double* ypcm, const double* zpcm,
                  const int* atomp, const double* co, const double* ecc12,
                  const double* ecc6, double alphal, const int* mapnl,
                  int ngrp, const int* grppt, double* ue, double* fpx,
                  double* fpy, double* fpz, double* stress, const int* nnlpp,
                  int* nnlpp1, long cap1, double rneigh, double rinn,
                  double rout, double rtolinn, double rtolout,
                  const double* gmass, int iz, const double* mass,
                  double massinfty, int lskip_ewald, int ewald, int nthreads,
                  const orc_variant* V, double* extra) {
  force_args A;
  memset(&A, 0, sizeof(A));
  A.V = (V && V->mode != 0) ? V : NULL;
  const int alch = A.V && A.V->mode == 2;
  A.ss_index = ss_index;
  A.xp0 = xp0;
  A.yp0 = yp0;
  A.zp0 = zp0;
  A.xpg = xpg;
  A.ypg = ypg;
  A.zpg = zpg;
  A.charge = charge;
  A.nbtype = nbtype;
  A.type = type;
  A.ma = ma;
  A.nato = nato;
  A.atomg = atomg;
  A.xpcm = xpcm;
  A.ypcm = ypcm;
  A.zpcm = zpcm;
  A.atomp = atomp;
  A.co = co;
  A.ecc12 = ecc12;
  A.ecc6 = ecc6;
  A.alphal = alphal;
  A.mapnl = mapnl;
  A.grppt = grppt;
  A.gmass = gmass;
  A.mass = mass;
  A.massinfty = massinfty;
  A.lskip_ewald = lskip_ewald;
  A.ewald = ewald;
  A.iz = iz;
  /* radii, force.f:145-167 (rinn0 uses rtolinn before it is reset) */
  A.rinn = rinn;
  A.r2inn = rinn * rinn;
  A.r2out = rout * rout;
  A.rinn0 = rinn + rtolinn;
  A.r2inn0 = A.rinn0 * A.rinn0;
  if (rinn < 1e-5) rtolinn = 0.0;
  A.rout0 = rout + rtolout;
  A.r2out0 = A.rout0 * A.rout0;
  A.r2neigh = (A.rinn0 + rneigh) * (A.rinn0 + rneigh);
  A.twrtpi = 2.0 / sqrt(PI_D);
  A.arsout1 = A.rout0 - 3.0 * rout;
  A.arsout2 = rtolout * rtolout * rtolout;
  A.arsinn1 = A.rinn0 - 3.0 * rinn;
  A.arsinn2 = rtolinn * rtolinn * rtolinn;

  long* mapoff = (long*)malloc(sizeof(long) * (nato + 1));
  {
    long o = 0;
    for (int a = 0; a < nato; a++) {
      mapoff[a] = o;
      o += mapnl[o] + 1;
    }
  }
  A.mapoff = mapoff;
  /* input list offsets: iz=1 walks the list group by group; iz=0 reads one
   * shared list from its start with mbeg = i+1 (force.f:243-263,826). */
  long* loff = (long*)malloc(sizeof(long) * (ngrp + 1));
  {
    long o = 0;
    for (int g = 0; g < ngrp; g++) {
      loff[g] = o;
      if (iz == 1) o += nnlpp[o] + 1;
    }
  }
  int maxlist = 0;
  for (int g = 0; g < ngrp; g++) {
    int c = nnlpp[loff[g]];
    if (c > maxlist) maxlist = c;
  }
  int want_next = rinn > 1.0e-5;
  int* nextcnt = (int*)calloc(ngrp, sizeof(int));
  int** nextlst = (int**)calloc(ngrp, sizeof(int*));

  double tot_conf[3] = {0, 0, 0}, tot_coul[3] = {0, 0, 0}, tot_st[9] = {0};
  double tot_seg = 0.0, tot_conf0[3] = {0, 0, 0}, tot_coul0[3] = {0, 0, 0};
  if (extra)
    for (int k = 0; k < 4; k++) extra[k] = 0.0;
  double* gfx = (double*)calloc(nato, sizeof(double));
  double* gfy = (double*)calloc(nato, sizeof(double));
  double* gfz = (double*)calloc(nato, sizeof(double));

#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
#endif
  {
    force_ws W;
    memset(&W, 0, sizeof(W));
    W.fx = (double*)calloc(nato, sizeof(double));
    W.fy = (double*)calloc(nato, sizeof(double));
    W.fz = (double*)calloc(nato, sizeof(double));
    W.maplg = (unsigned char*)malloc(nato);
    W.mapag = (unsigned char*)malloc(ngrp);
    memset(W.maplg, 1, nato);
    memset(W.mapag, 1, ngrp);
    int cap = maxlist + 1;
    W.index0 = (int*)malloc(sizeof(int) * cap);
    W.index1 = (int*)malloc(sizeof(int) * cap);
    W.nlist_out = (int*)malloc(sizeof(int) * cap);
    W.drs = (double*)malloc(sizeof(double) * cap);
    double** dp[] = {&W.xmap0, &W.ymap0, &W.zmap0, &W.xmap1, &W.ymap1,
                     &W.zmap1, &W.xmap2, &W.ymap2, &W.zmap2, &W.cmap2,
                     &W.swrs,  &W.dswrs, &W.xmap3, &W.ymap3, &W.zmap3};
    for (unsigned k = 0; k < sizeof(dp) / sizeof(dp[0]); k++)
      *dp[k] = (double*)malloc(sizeof(double) * cap);
#ifdef _OPENMP
    /* cache_line ownership: chunks of 16 groups dealt round-robin
     * (src/omp_integr.f90:207-232) */
#pragma omp for schedule(static, 16)
#endif
    for (int i = 0; i < ngrp; i++) {
      const int* lst = nnlpp + loff[i] + 1;
      int m = nnlpp[loff[i]];
      int mbeg = (iz == 0) ? i + 1 : 0;
      int map = alch ? force_group_alch(&A, &W, i, lst, m, mbeg)
                     : force_group(&A, &W, i, lst, m, mbeg);
      if (want_next) {
        nextcnt[i] = map;
        nextlst[i] = (int*)malloc(sizeof(int) * (map > 0 ? map : 1));
        memcpy(nextlst[i], W.nlist_out, sizeof(int) * map);
      }
    }
#ifdef _OPENMP
#pragma omp critical
#endif
    {
      for (int a = 0; a < nato; a++) {
        gfx[a] += W.fx[a];
        gfy[a] += W.fy[a];
        gfz[a] += W.fz[a];
      }
      for (int k = 0; k < 3; k++) {
        tot_conf[k] += W.uconf[k];
        tot_coul[k] += W.ucoul[k];
      }
      for (int k = 0; k < 9; k++) tot_st[k] += W.st[k];
      tot_seg += W.seg_ene;
      for (int k = 0; k < 3; k++) {
        tot_conf0[k] += W.uconf0[k];
        tot_coul0[k] += W.ucoul0[k];
      }
    }
    free(W.fx);
    free(W.fy);
    free(W.fz);
    free(W.maplg);
    free(W.mapag);
    free(W.index0);
    free(W.index1);
    free(W.nlist_out);
    free(W.drs);
    for (unsigned k = 0; k < sizeof(dp) / sizeof(dp[0]); k++) free(*dp[k]);
  }
  long ncount1 = 0;
  if (want_next) {
    for (int i = 0; i < ngrp; i++) {
      if (ncount1 + nextcnt[i] + 1 > cap1) {
        ncount1 = -1;
        break;
      }
      nnlpp1[ncount1] = nextcnt[i];
      memcpy(nnlpp1 + ncount1 + 1, nextlst[i], sizeof(int) * nextcnt[i]);
      ncount1 += nextcnt[i] + 1;
    }
    for (int i = 0; i < ngrp; i++) free(nextlst[i]);
  }
  free(nextlst);
  free(nextcnt);
  int forces_on = !(iz == 0 || A.rinn0 >= rout);
  if (forces_on) { /* force.f:841-870 */
    for (int a = 0; a < nato; a++) {
      fpx[a] += gfx[a];
      fpy[a] += gfy[a];
      fpz[a] += gfz[a];
    }
    ue[0] = tot_conf[0];
    ue[1] = tot_conf[2];
    ue[2] = tot_conf[1];
    ue[3] = tot_coul[0];
    ue[4] = tot_coul[2];
    ue[5] = tot_coul[1];
    if (extra) {
      extra[0] = tot_seg;
      /* src/force_alchemy.f:683-688 */
      double dwrk = 0.0;
      for (int k = 0; k < 3; k++) {
        double auxa = tot_coul[k] - tot_coul0[k];
        double auxb = tot_conf[k] - tot_conf0[k];
        dwrk = dwrk + auxa + auxb;
      }
      extra[1] = alch ? dwrk : 0.0;
      extra[2] = tot_conf0[0] + tot_conf0[1] + tot_conf0[2];
      extra[3] = tot_coul0[0] + tot_coul0[1] + tot_coul0[2];
    }
    /* st(i,j) row-major in tot_st[3*i+j]; stress(i,j) += sum_k st(i,k) co(j,k) */
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        for (int k = 0; k < 3; k++)
          stress[a + 3 * b] += tot_st[3 * a + k] * co[b + 3 * k];
  }
  free(gfx);
  free(gfy);
  free(gfz);
  free(mapoff);
  free(loff);
  return want_next ? ncount1 : 0;
}

/* ------------------------------------------------------------------- PME */

/* fill_bspline/init/one_pass/diff, src/pme_fftw3.f90:518-576 */
void orc_fill_bspline(double w, int order, double* c, double* d) {
  c[order - 1] = 0.0;
  c[1] = w;
  c[0] = 1.0 - w;
  for (int k = 3; k <= order - 1; k++) {
    double div = 1.0 / (k - 1);
    c[k - 1] = div * w * c[k - 2];
    for (int j = 1; j <= k - 2; j++)
      c[k - j - 1] = div * ((w + j) * c[k - j - 2] + (k - j - w) * c[k - j - 1]);
    c[0] = div * (1 - w) * c[0];
  }
  d[0] = -c[0];
  for (int j = 2; j <= order; j++) d[j - 1] = c[j - 2] - c[j - 1];
  {
    int k = order;
    double div = 1.0 / (k - 1);
    c[k - 1] = div * w * c[k - 2];
    for (int j = 1; j <= k - 2; j++)
      c[k - j - 1] = div * ((w + j) * c[k - j - 2] + (k - j - w) * c[k - j - 1]);
    c[0] = div * (1 - w) * c[0];
  }
}

/* DFTMOD, src/pme_fftw3.f90:202-229.  twopi is 2.d0 times a default-real
 * literal of pi, i.e. 2*(float)pi. */
static void dftmod(double* bsp_mod, const double* bsp_arr, int nfft) {
  double twopi = 2.0 * (double)3.14159265358979323846f;
  double tiny = 1.0e-7;
  for (int k = 1; k <= nfft; k++) {
    double s1 = 0, s2 = 0;
    for (int j = 1; j <= nfft; j++) {
      double arg = twopi * (k - 1) * (j - 1) / nfft;
      s1 += bsp_arr[j - 1] * cos(arg);
      s2 += bsp_arr[j - 1] * sin(arg);
    }
    bsp_mod[k - 1] = s1 * s1 + s2 * s2;
  }
  for (int k = 1; k <= nfft; k++)
    if (bsp_mod[k - 1] < tiny) {
      /* the reference reads bsp_mod(0)/bsp_mod(nfft+1) out of bounds at the
       * ends; a B-spline modulus is never tiny there (k=1 is the sum of the
       * weights, 1), so only interior points reach this average. */
      double lo = (k >= 2) ? bsp_mod[k - 2] : bsp_mod[nfft - 1];
      double hi = (k <= nfft - 1) ? bsp_mod[k] : bsp_mod[0];
      bsp_mod[k - 1] = 0.5 * (lo + hi);
    }
}

/* load_bsp_moduli, src/pme_fftw3.f90:165-200 */
void orc_load_bsp_moduli(double* m1, double* m2, double* m3, int nfft1,
                         int nfft2, int nfft3, int order) {
  int maxn = nfft1 > nfft2 ? nfft1 : nfft2;
  if (nfft3 > maxn) maxn = nfft3;
  double arr[32], darr[32];
  double* bsp_arr = (double*)calloc(maxn + 1, sizeof(double));
  orc_fill_bspline(0.0, order, arr, darr);
  for (int i = 2; i <= order + 1; i++) bsp_arr[i - 1] = arr[i - 2];
  dftmod(m1, bsp_arr, nfft1);
  dftmod(m2, bsp_arr, nfft2);
  dftmod(m3, bsp_arr, nfft3);
  free(bsp_arr);
}

/* Mixed-radix complex DFT (decimation in time over the smallest prime
 * factor, direct sums for that factor), double precision, twiddles from
 * cos/sin.  sign = -1 forward, +1 backward, unnormalised. */
static void fft_level(int n, const double* in, long istride, double* out,
                      int sign) {
  if (n == 1) {
    out[0] = in[0];
    out[1] = in[1];
    return;
  }
  int p = 2;
  while (n % p) p++;
  int m = n / p;
  double* sub = (double*)malloc(sizeof(double) * 2 * n);
  for (int r = 0; r < p; r++)
    fft_level(m, in + 2 * r * istride, istride * p, sub + 2 * r * m, sign);
  for (int k = 0; k < m; k++)
    for (int q = 0; q < p; q++) {
      int kk = k + q * m;
      double sr = 0, si = 0;
      for (int r = 0; r < p; r++) {
        double ang = sign * 2.0 * PI_D * (double)(((long)r * kk) % n) / n;
        double c = cos(ang), s = sin(ang);
        double xr = sub[2 * (r * m + k)], xi = sub[2 * (r * m + k) + 1];
        sr += xr * c - xi * s;
        si += xr * s + xi * c;
      }
      out[2 * kk] = sr;
      out[2 * kk + 1] = si;
    }
  free(sub);
}

static void fft1d(int n, double* data /* 2n interleaved */, int sign) {
  double* in = (double*)malloc(sizeof(double) * 2 * n);
  memcpy(in, data, sizeof(double) * 2 * n);
  fft_level(n, in, 1, data, sign);
  free(in);
}

/* 1-D transform exported for the tests */
void orc_fft1d(int n, double* data, int sign) { fft1d(n, data, sign); }

void orc_fft3d_r2c(int n1, int n2, int n3, const double* Q, double* FQ) {
  int h1 = n1 / 2 + 1;
  int nmax = n1 > n2 ? n1 : n2;
  if (n3 > nmax) nmax = n3;
  double* line = (double*)malloc(sizeof(double) * 2 * nmax);
  for (int k = 0; k < n3; k++)
    for (int j = 0; j < n2; j++) {
      for (int i = 0; i < n1; i++) {
        line[2 * i] = Q[i + (long)n1 * (j + (long)n2 * k)];
        line[2 * i + 1] = 0.0;
      }
      fft1d(n1, line, -1);
      for (int i = 0; i < h1; i++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        FQ[o] = line[2 * i];
        FQ[o + 1] = line[2 * i + 1];
      }
    }
  for (int k = 0; k < n3; k++)
    for (int i = 0; i < h1; i++) {
      for (int j = 0; j < n2; j++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        line[2 * j] = FQ[o];
        line[2 * j + 1] = FQ[o + 1];
      }
      fft1d(n2, line, -1);
      for (int j = 0; j < n2; j++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        FQ[o] = line[2 * j];
        FQ[o + 1] = line[2 * j + 1];
      }
    }
  for (int j = 0; j < n2; j++)
    for (int i = 0; i < h1; i++) {
      for (int k = 0; k < n3; k++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        line[2 * k] = FQ[o];
        line[2 * k + 1] = FQ[o + 1];
      }
      fft1d(n3, line, -1);
      for (int k = 0; k < n3; k++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        FQ[o] = line[2 * k];
        FQ[o + 1] = line[2 * k + 1];
      }
    }
  free(line);
}

void orc_fft3d_c2r(int n1, int n2, int n3, const double* FQin, double* Q) {
  int h1 = n1 / 2 + 1;
  long nh = (long)h1 * n2 * n3;
  double* FQ = (double*)malloc(sizeof(double) * 2 * nh);
  memcpy(FQ, FQin, sizeof(double) * 2 * nh);
  int nmax = n1 > n2 ? n1 : n2;
  if (n3 > nmax) nmax = n3;
  double* line = (double*)malloc(sizeof(double) * 2 * nmax);
  for (int j = 0; j < n2; j++)
    for (int i = 0; i < h1; i++) {
      for (int k = 0; k < n3; k++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        line[2 * k] = FQ[o];
        line[2 * k + 1] = FQ[o + 1];
      }
      fft1d(n3, line, +1);
      for (int k = 0; k < n3; k++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        FQ[o] = line[2 * k];
        FQ[o + 1] = line[2 * k + 1];
      }
    }
  for (int k = 0; k < n3; k++)
    for (int i = 0; i < h1; i++) {
      for (int j = 0; j < n2; j++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        line[2 * j] = FQ[o];
        line[2 * j + 1] = FQ[o + 1];
      }
      fft1d(n2, line, +1);
      for (int j = 0; j < n2; j++) {
        long o = 2 * (i + (long)h1 * (j + (long)n2 * k));
        FQ[o] = line[2 * j];
        FQ[o + 1] = line[2 * j + 1];
      }
    }
  for (int k = 0; k < n3; k++)
    for (int j = 0; j < n2; j++) {
      for (int i = 0; i < n1; i++) {
        int src = (i < h1) ? i : n1 - i;
        long o = 2 * (src + (long)h1 * (j + (long)n2 * k));
        line[2 * i] = FQ[o];
        line[2 * i + 1] = (i < h1) ? FQ[o + 1] : -FQ[o + 1];
      }
      fft1d(n1, line, +1);
      for (int i = 0; i < n1; i++) Q[i + (long)n1 * (j + (long)n2 * k)] = line[2 * i];
    }
  free(line);
  free(FQ);
}

/* scalar_sum, FFTW branch, src/scalar_sum.f:2-135.  pi there is a
 * default-real literal: (float)pi widened to double. */
void orc_scalar_sum(double* FQ, double ewaldcof, double volume,
                    const double* recip, const double* bsp_mod1,
                    const double* bsp_mod2, const double* bsp_mod3, int nfft1,
                    int nfft2, int nfft3, double* eer, double* vir,
                    double rkcut) {
  int ndim1 = 1 + nfft1 / 2;
  long indtop = (long)ndim1 * nfft2 * nfft3;
  double pi = (double)3.14159265358979323846f;
  double rkcut2 = 0.25 * rkcut * rkcut / (pi * pi);
  double fac = pi * pi / (ewaldcof * ewaldcof);
  long nff = (long)ndim1 * nfft2;
  int nf1 = nfft1 / 2;
  if (2 * nf1 < nfft1) nf1++;
  int nf2 = nfft2 / 2;
  if (2 * nf2 < nfft2) nf2++;
  int nf3 = nfft3 / 2;
  if (2 * nf3 < nfft3) nf3++;
  double energy = 0.0;
  double v11 = 0, v22 = 0, v33 = 0, v12 = 0, v13 = 0, v23 = 0;
  for (long ind = 1; ind <= indtop - 1; ind++) {
    int k3 = (int)(ind / nff) + 1;
    long jnd = ind - (long)(k3 - 1) * nff;
    int k2 = (int)(jnd / ndim1) + 1;
    int k1 = (int)(jnd - (long)(k2 - 1) * ndim1) + 1;
    int m1 = k1 - 1;
    if (k1 > nf1) m1 = k1 - 1 - nfft1;
    int m2 = k2 - 1;
    if (k2 > nf2) m2 = k2 - 1 - nfft2;
    int m3 = k3 - 1;
    if (k3 > nf3) m3 = k3 - 1 - nfft3;
    double mh1 = recip[0] * m1 + recip[3] * m2 + recip[6] * m3;
    double mh2 = recip[1] * m1 + recip[4] * m2 + recip[7] * m3;
    double mh3 = recip[2] * m1 + recip[5] * m2 + recip[8] * m3;
    double msq = mh1 * mh1 + mh2 * mh2 + mh3 * mh3;
    double eterm;
    double* q = FQ + 2 * ind;
    if (msq > rkcut2) {
      eterm = 0.0;
    } else {
      double denom = pi * volume * bsp_mod1[k1 - 1] * bsp_mod2[k2 - 1] *
                     bsp_mod3[k3 - 1] * msq;
      eterm = exp(-fac * msq) / denom;
      double vterm = 2.0 * (fac * msq + 1.0) / msq;
      double q2 = q[0] * q[0] + q[1] * q[1];
      double struc2, vvir, fac12, fac13, fac23;
      if (k1 == 1 || (k1 == ndim1 && nfft1 % 2 == 0)) {
        struc2 = eterm * q2;
        vvir = struc2 * vterm;
        fac12 = fac13 = fac23 = 1.0;
      } else {
        struc2 = 2.0 * eterm * q2;
        vvir = struc2 * vterm;
        fac12 = (mh1 * mh2 < 0.0 && k2 <= ndim1) ? 0.0 : 1.0;
        fac13 = (mh1 * mh3 < 0.0 && k3 <= ndim1) ? 0.0 : 1.0;
        int neg = mh2 * mh3 < 0.0;
        if (k2 <= ndim1 && k3 <= ndim1)
          fac23 = neg ? 0.0 : 1.0;
        else if (k2 > ndim1 && k3 <= ndim1)
          fac23 = neg ? 1.0 : 0.0;
        else if (k3 > ndim1 && k2 <= ndim1)
          fac23 = neg ? 1.0 : 0.0;
        else
          fac23 = neg ? 0.0 : 1.0;
      }
      energy += struc2;
      v11 += struc2 * (vterm * mh1 * mh1 - 1.0);
      v22 += struc2 * (vterm * mh2 * mh2 - 1.0);
      v33 += struc2 * (vterm * mh3 * mh3 - 1.0);
      v12 += vvir * mh1 * mh2 * fac12;
      v13 += vvir * mh1 * mh3 * fac13;
      v23 += vvir * mh2 * mh3 * fac23;
    }
    q[0] *= eterm;
    q[1] *= eterm;
  }
  *eer = 0.5 * energy;
  vir[0] = 0.5 * v11;
  vir[4] = 0.5 * v22;
  vir[8] = 0.5 * v33;
  vir[3] = vir[1] = 0.5 * v12;
  vir[6] = vir[2] = 0.5 * v13;
  vir[7] = vir[5] = 0.5 * v23;
}

/* grid index of fill_charge_grid/grad_sum, src/pme_fftw3.f90:272-290:
 * k = k0 + 1 + (n - isign(n,k0))/2 (1-based).  When a fractional coordinate
 * sits exactly at n (w - anint(w) = 0.5) the reference indexes n+1, past the
 * end of that dimension; that measure-zero case is wrapped here. */
static inline int grid_index(int k0, int n) {
  int k = (k0 >= 0) ? k0 : k0 + n; /* 0-based */
  if (k >= n) k -= n;
  return k;
}

void orc_do_pmesh_kspace(int numatoms, const double* x, const double* y,
                         const double* z, const double* charge,
                         const double* recip, double volume,
                         double ewald_coeff, int order, int nfft1, int nfft2,
                         int nfft3, double* eer, double* dx, double* dy,
                         double* dz, double* vir, double rkcut, int nthreads) {
  (void)nthreads;
  double* fr1 = (double*)malloc(sizeof(double) * numatoms);
  double* fr2 = (double*)malloc(sizeof(double) * numatoms);
  double* fr3 = (double*)malloc(sizeof(double) * numatoms);
  double* th1 = (double*)malloc(sizeof(double) * numatoms * order);
  double* th2 = (double*)malloc(sizeof(double) * numatoms * order);
  double* th3 = (double*)malloc(sizeof(double) * numatoms * order);
  double* dth1 = (double*)malloc(sizeof(double) * numatoms * order);
  double* dth2 = (double*)malloc(sizeof(double) * numatoms * order);
  double* dth3 = (double*)malloc(sizeof(double) * numatoms * order);
  long ng = (long)nfft1 * nfft2 * nfft3;
  long nh = (long)(nfft1 / 2 + 1) * nfft2 * nfft3;
  double* Q = (double*)calloc(ng, sizeof(double));
  double* FQ = (double*)malloc(sizeof(double) * 2 * nh);
  double* b1 = (double*)malloc(sizeof(double) * nfft1);
  double* b2 = (double*)malloc(sizeof(double) * nfft2);
  double* b3 = (double*)malloc(sizeof(double) * nfft3);
  orc_load_bsp_moduli(b1, b2, b3, nfft1, nfft2, nfft3, order);
  /* get_scaled_fractionals, pme_fftw3.f90:132-163 */
  for (int n = 0; n < numatoms; n++) {
    double w = x[n] * recip[0] + y[n] * recip[1] + z[n] * recip[2];
    fr1[n] = nfft1 * (w - round(w) + 0.5);
    w = x[n] * recip[3] + y[n] * recip[4] + z[n] * recip[5];
    fr2[n] = nfft2 * (w - round(w) + 0.5);
    w = x[n] * recip[6] + y[n] * recip[7] + z[n] * recip[8];
    fr3[n] = nfft3 * (w - round(w) + 0.5);
  }
  /* get_bspline_coeffs, pme_fftw3.f90:487-512 */
  for (int n = 0; n < numatoms; n++) {
    orc_fill_bspline(fr1[n] - (int)fr1[n], order, th1 + n * order, dth1 + n * order);
    orc_fill_bspline(fr2[n] - (int)fr2[n], order, th2 + n * order, dth2 + n * order);
    orc_fill_bspline(fr3[n] - (int)fr3[n], order, th3 + n * order, dth3 + n * order);
  }
  /* fill_charge_grid, pme_fftw3.f90:264-294 */
  for (int n = 0; n < numatoms; n++) {
    int k0 = (int)fr3[n] - order;
    for (int i3 = 0; i3 < order; i3++) {
      k0++;
      int k = grid_index(k0, nfft3);
      int j0 = (int)fr2[n] - order;
      for (int i2 = 0; i2 < order; i2++) {
        j0++;
        int j = grid_index(j0, nfft2);
        double prod = th2[n * order + i2] * th3[n * order + i3] * charge[n];
        int i0 = (int)fr1[n] - order;
        for (int i1 = 0; i1 < order; i1++) {
          i0++;
          int i = grid_index(i0, nfft1);
          Q[i + (long)nfft1 * (j + (long)nfft2 * k)] += th1[n * order + i1] * prod;
        }
      }
    }
  }
  orc_fft3d_r2c(nfft1, nfft2, nfft3, Q, FQ);
  orc_scalar_sum(FQ, ewald_coeff, volume, recip, b1, b2, b3, nfft1, nfft2,
                 nfft3, eer, vir, rkcut);
  orc_fft3d_c2r(nfft1, nfft2, nfft3, FQ, Q);
  /* grad_sum, pme_fftw3.f90:310-372 */
  for (int n = 0; n < numatoms; n++) {
    double f1 = 0, f2 = 0, f3 = 0;
    int k0 = (int)fr3[n] - order;
    for (int i3 = 0; i3 < order; i3++) {
      k0++;
      int k = grid_index(k0, nfft3);
      int j0 = (int)fr2[n] - order;
      for (int i2 = 0; i2 < order; i2++) {
        j0++;
        int j = grid_index(j0, nfft2);
        int i0 = (int)fr1[n] - order;
        for (int i1 = 0; i1 < order; i1++) {
          i0++;
          int i = grid_index(i0, nfft1);
          double term = charge[n] * Q[i + (long)nfft1 * (j + (long)nfft2 * k)];
          f1 -= nfft1 * term * dth1[n * order + i1] * th2[n * order + i2] * th3[n * order + i3];
          f2 -= nfft2 * term * th1[n * order + i1] * dth2[n * order + i2] * th3[n * order + i3];
          f3 -= nfft3 * term * th1[n * order + i1] * th2[n * order + i2] * dth3[n * order + i3];
        }
      }
    }
    dx[n] += recip[0] * f1 + recip[3] * f2 + recip[6] * f3;
    dy[n] += recip[1] * f1 + recip[4] * f2 + recip[7] * f3;
    dz[n] += recip[2] * f1 + recip[5] * f2 + recip[8] * f3;
  }
  free(fr1);
  free(fr2);
  free(fr3);
  free(th1);
  free(th2);
  free(th3);
  free(dth1);
  free(dth2);
  free(dth3);
  free(Q);
  free(FQ);
  free(b1);
  free(b2);
  free(b3);
}

/* fft_pme, src/fft_pme.f:30-112 */
void orc_fft_pme(int ntap, const double* xp, const double* yp, const double* zp,
                 const double* xpcm, const double* ypcm, const double* zpcm,
                 const double* pmechg, const double* co, const double* oc,
                 double volume, double alphal, int order, int nfft1, int nfft2,
                 int nfft3, double* eer, double* fpx, double* fpy, double* fpz,
                 double* stressc, const int* atomp, int pressure, double rkcut,
                 int nthreads) {
  double* x = (double*)malloc(sizeof(double) * ntap);
  double* y = (double*)malloc(sizeof(double) * ntap);
  double* z = (double*)malloc(sizeof(double) * ntap);
  double* fx = (double*)calloc(ntap, sizeof(double));
  double* fy = (double*)calloc(ntap, sizeof(double));
  double* fz = (double*)calloc(ntap, sizeof(double));
  orc_change_frame(co, oc, 1, ntap, xp, yp, zp, x, y, z);
  double recip[9], vir[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) recip[i + 3 * j] = 0.5 * oc[j + 3 * i];
  orc_do_pmesh_kspace(ntap, x, y, z, pmechg, recip, volume, alphal, order,
                      nfft1, nfft2, nfft3, eer, fx, fy, fz, vir, rkcut,
                      nthreads);
  if (pressure) {
    double stc[9] = {0};
    for (int i = 0; i < ntap; i++) {
      int j = atomp[i] - 1;
      double sx = xp[i] - xpcm[j], sy = yp[i] - ypcm[j], sz = zp[i] - zpcm[j];
      double gx = sx * co[0] + sy * co[3] + sz * co[6];
      double gy = sx * co[1] + sy * co[4] + sz * co[7];
      double gz = sx * co[2] + sy * co[5] + sz * co[8];
      stc[0] -= gx * fx[i];
      stc[1] -= gy * fx[i];
      stc[2] -= gz * fx[i];
      stc[3] -= gx * fy[i];
      stc[4] -= gy * fy[i];
      stc[5] -= gz * fy[i];
      stc[6] -= gx * fz[i];
      stc[7] -= gy * fz[i];
      stc[8] -= gz * fz[i];
    }
    /* stressc(a,b) -= vir(a,b) ; += stc(row a, col b) */
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        stressc[a + 3 * b] += -vir[a + 3 * b] + stc[3 * a + b];
  }
  for (int i = 0; i < ntap; i++) {
    fpx[i] += fx[i];
    fpy[i] += fy[i];
    fpz[i] += fz[i];
  }
  free(x);
  free(y);
  free(z);
  free(fx);
  free(fy);
  free(fz);
}

/* ferrf, src/ferrf.f:53-151 (iz=1) and :194-230 (iz=0), erf_corr false */
void orc_ferrf(const int* ss_index, double alphal, const double* charge,
               double fudge, const double* x0, const double* y0,
               const double* z0, int iz, const int* list, int nlist,
               double* fs, double* fpx, double* fpy, double* fpz) {
  double twrtpi = 2.0 / sqrt(PI_D);
  double fsr[2] = {0, 0};
  for (int i = 0; i < nlist; i++) {
    int ia = list[2 * i] - 1, ib = list[2 * i + 1] - 1;
    int type = ss_index[ia];
    double furpar = (iz == 1 ? fudge : 1.0) * charge[ia] * charge[ib];
    double xab = x0[ia] - x0[ib], yab = y0[ia] - y0[ib], zab = z0[ia] - z0[ib];
    double rsq = xab * xab + yab * yab + zab * zab;
    double rsp = sqrt(rsq);
    double alphar = alphal * rsp;
    double qt = 1.0 / (1.0 + AS_QP * alphar);
    double expcst = exp(-alphar * alphar);
    double erfcst =
        ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt *
        expcst;
    double erfst = 1.0 - erfcst;
    fsr[type - 1] -= furpar * erfst / rsp;
    if (iz == 1) {
      double qforce = -furpar * (erfst - twrtpi * alphar * expcst) / (rsp * rsq);
      fpx[ia] += qforce * xab;
      fpy[ia] += qforce * yab;
      fpz[ia] += qforce * zab;
      fpx[ib] -= qforce * xab;
      fpy[ib] -= qforce * yab;
      fpz[ib] -= qforce * zab;
    }
  }
  fs[0] = fsr[0];
  fs[1] = fsr[1];
}

/* cself, src/cself.f:44-60 */
void orc_cself(const int* ss_index, const double* charge, int nato,
               double alphal, double kcut, double* self_slt,
               double* self_slv) {
  double f[2] = {0, 0};
  for (int n = 0; n < nato; n++) f[ss_index[n] - 1] += charge[n] * charge[n];
  for (int n = 0; n < 2; n++) {
    double erfcst = orc_erfc_as(kcut / (2.0 * alphal));
    f[n] = -f[n] * alphal / sqrt(PI_D) * (1.0 - erfcst);
  }
  *self_slt = f[0];
  *self_slv = f[1];
}

/* fnb14, src/fnb14.f:86-209 */
void orc_fnb14(const int* ss_index, const double* xp0, const double* yp0,
               const double* zp0, const double* charge, int nato,
               const double* ecc12, const double* ecc6, int cut, int ewald,
               double alphal, const int* int14, int int14p,
               const int* type14, double fudge, double lj_fudge, double* fpx,
               double* fpy, double* fpz, double* ue) {
  (void)nato;
  double uconf[2] = {0, 0}, ucoul[2] = {0, 0};
  double twrtpi = 2.0 / sqrt(PI_D);
  int bare = (!ewald || !cut);
  for (int i = 0; i < int14p; i++) {
    int i1 = int14[2 * i] - 1, i2 = int14[2 * i + 1] - 1;
    int type = ss_index[i1];
    int lij = type14[i] - 1;
    double xa = xp0[i1] - xp0[i2], ya = yp0[i1] - yp0[i2], za = zp0[i1] - zp0[i2];
    double rsq = xa * xa + ya * ya + za * za;
    double rsp = sqrt(rsq);
    double rsqi = 1.0 / rsq;
    double r6 = rsqi * rsqi * rsqi;
    double r12 = r6 * r6;
    double ssvir = 12.0 * ecc12[lij] * r12 - 6.0 * ecc6[lij] * r6;
    double qforce;
    if (bare) {
      qforce = lj_fudge * ssvir * rsqi;
      uconf[type - 1] += lj_fudge * (ecc12[lij] * r12 - ecc6[lij] * r6);
      double sv = fudge * charge[i1] * charge[i2] / rsp;
      ucoul[type - 1] += sv;
      qforce += sv * rsqi;
    } else {
      double rspqi = rsqi / rsp;
      uconf[type - 1] += lj_fudge * (ecc12[lij] * r12 - ecc6[lij] * r6);
      double alphar = alphal * rsp;
      double qt = 1.0 / (1.0 + AS_QP * alphar);
      double expcst = exp(-alphar * alphar);
      double erfcst =
          ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) *
          qt * expcst;
      double furpar = fudge * charge[i1] * charge[i2];
      ucoul[type - 1] += furpar * erfcst / rsp;
      qforce = lj_fudge * ssvir * rsqi +
               furpar * (erfcst + twrtpi * alphar * expcst) * rspqi;
    }
    fpx[i1] += qforce * xa;
    fpy[i1] += qforce * ya;
    fpz[i1] += qforce * za;
    fpx[i2] -= qforce * xa;
    fpy[i2] -= qforce * ya;
    fpz[i2] -= qforce * za;
  }
  ue[0] = uconf[0];
  ue[1] = uconf[1];
  ue[2] = ucoul[0];
  ue[3] = ucoul[1];
}

/* fnbgrp, src/fnbgrp.f:96-202; lij = max*(max-1)/2 + min of the LJ types */
void orc_fnbgrp(const int* ss_index, const double* xp0, const double* yp0,
                const double* zp0, const double* charge, const int* type,
                const double* ecc12, const double* ecc6, int ewald,
                double alphal, const int* ingrp, int ingrpp, double* fpx,
                double* fpy, double* fpz, double* ue) {
  double uconf[2] = {0, 0}, ucoul[2] = {0, 0};
  double twrtpi = 2.0 / sqrt(PI_D);
  for (int i = 0; i < ingrpp; i++) {
    int i1 = ingrp[2 * i] - 1, i2 = ingrp[2 * i + 1] - 1;
    int typei = ss_index[i1];
    int lj = type[i1] > type[i2] ? type[i1] : type[i2];
    int li = type[i1] > type[i2] ? type[i2] : type[i1];
    int lij = lj * (lj - 1) / 2 + li - 1;
    double xa = xp0[i1] - xp0[i2], ya = yp0[i1] - yp0[i2], za = zp0[i1] - zp0[i2];
    double rsq = xa * xa + ya * ya + za * za;
    double rsp = sqrt(rsq);
    double rsqi = 1.0 / rsq;
    double r6 = rsqi * rsqi * rsqi;
    double r12 = r6 * r6;
    double ssvir = 12.0 * ecc12[lij] * r12 - 6.0 * ecc6[lij] * r6;
    double qforce = ssvir * rsqi;
    uconf[typei - 1] += ecc12[lij] * r12 - ecc6[lij] * r6;
    if (!ewald) {
      double sv = charge[i1] * charge[i2] / rsp;
      ucoul[typei - 1] += sv;
      qforce += sv * rsqi;
    } else {
      double rspqi = rsqi / rsp;
      double alphar = alphal * rsp;
      double qt = 1.0 / (1.0 + AS_QP * alphar);
      double expcst = exp(-alphar * alphar);
      double erfcst =
          ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) *
          qt * expcst;
      double furpar = charge[i1] * charge[i2];
      ucoul[typei - 1] += furpar * erfcst / rsp;
      qforce += furpar * (erfcst + twrtpi * alphar * expcst) * rspqi;
    }
    fpx[i1] += qforce * xa;
    fpy[i1] += qforce * ya;
    fpz[i1] += qforce * za;
    fpx[i2] -= qforce * xa;
    fpy[i2] -= qforce * ya;
    fpz[i2] -= qforce * za;
  }
  ue[0] = uconf[0];
  ue[1] = uconf[1];
  ue[2] = ucoul[0];
  ue[3] = ucoul[1];
}

/* The per-atom lambdas of ORAC's alchemical species (src/mtsmd.f:746-754,
 * src/initialize_lambda.f:30-52): added atoms carry ladd, removed atoms
 * -lrm, all others 0; the coupling of an atom is 1 - |lambda|. */
void orc_alch_atom_lambdas(int nato, const int* ss_alchemy, double ladd, double lrm, double* lam) {
  for (int i = 0; i < nato; i++) lam[i] = ss_alchemy[i] == 2 ? ladd : (ss_alchemy[i] == -2 ? -lrm : 0.0);
}

/* listqq of src/initialize_lambda.f:62-139: every pair of alchemical atoms
 * (added or removed) that is no 1-2 (bond or constraint), 1-3 or 1-4 pair,
 * as (ia, ib, facQ) 1-based, facQ = 1 for atoms of one species, 0 for an
 * added-removed pair.  The excluded pairs come as one 1-based list of
 * nexcl pairs.  Returns the number of entries written (at most cap). */
int orc_alch_listqq(int nato, const int* ss_alchemy, const int* excl, int nexcl, int* out3, int cap) {
  int nat = 0;
  for (int i = 0; i < nato; i++) nat += (ss_alchemy[i] == 2 || ss_alchemy[i] == -2);
  int* iat = (int*)malloc(sizeof(int) * (nat > 0 ? nat : 1));
  int k = 0;
  /* ORAC's order: added atoms first, then removed ones */
  for (int i = 0; i < nato; i++)
    if (ss_alchemy[i] == 2) iat[k++] = i + 1;
  for (int i = 0; i < nato; i++)
    if (ss_alchemy[i] == -2) iat[k++] = i + 1;
  int n = 0;
  for (int a = 0; a < nat - 1; a++)
    for (int b = a + 1; b < nat; b++) {
      const int ia = iat[a], ib = iat[b];
      int skip = 0;
      for (int l = 0; l < nexcl && !skip; l++)
        skip = (excl[2 * l] == ia && excl[2 * l + 1] == ib) || (excl[2 * l] == ib && excl[2 * l + 1] == ia);
      if (skip) continue;
      if (n < cap) {
        out3[3 * n] = ia;
        out3[3 * n + 1] = ib;
        out3[3 * n + 2] = ss_alchemy[ia - 1] == ss_alchemy[ib - 1] ? 1 : 0;
      }
      n++;
    }
  free(iat);
  return n;
}

/* ferrf_alchemy_add, src/ferrf_alchemy_add.f (the branch without the erf
 * tables, ORAC's default): the reciprocal sum of the scaled charges
 * (1 - |lq|) Q gives every listqq pair (1-|lq_a|)(1-|lq_b|) Q_a Q_b erf/r;
 * this subtracts factl Q_a Q_b erf(alpha r)/r with factl = that product -
 * facQ, so that atoms of one species keep their full Coulomb (facQ 1) and
 * added and removed atoms do not see each other (facQ 0).  With intramol
 * the pairs of one species are skipped.  fs receives the energies (solute,
 * solvent), *dwrk the work U(lambda) - U(lambda0). */
void orc_ferrf_alchemy_add(const int* ss_index, double alphal, const double* charge, const double* lambdaq,
                           const double* lambdaq0, const double* x0, const double* y0, const double* z0,
                           const int* list3, int nlist, int intramol, double* fs, double* dwrk, double* fpx,
                           double* fpy, double* fpz) {
  double twrtpi = 2.0 / sqrt(PI_D);
  double fsr[2] = {0, 0}, en0 = 0.0;
  for (int i = 0; i < nlist; i++) {
    int ia = list3[3 * i] - 1, ib = list3[3 * i + 1] - 1;
    double facq = (double)list3[3 * i + 2];
    if (intramol && list3[3 * i + 2] != 0) continue;
    int type = ss_index[ia];
    double factl = (1.0 - fabs(lambdaq[ia])) * (1.0 - fabs(lambdaq[ib])) - facq;
    double factl0 = (1.0 - fabs(lambdaq0[ia])) * (1.0 - fabs(lambdaq0[ib])) - facq;
    double furpar = factl * charge[ia] * charge[ib];
    double furpar0 = factl0 * charge[ia] * charge[ib];
    double xab = x0[ia] - x0[ib], yab = y0[ia] - y0[ib], zab = z0[ia] - z0[ib];
    double rsq = xab * xab + yab * yab + zab * zab;
    double rsp = sqrt(rsq);
    double alphar = alphal * rsp;
    double qt = 1.0 / (1.0 + AS_QP * alphar);
    double expcst = exp(-alphar * alphar);
    double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
    double erfst = 1.0 - erfcst;
    double qforce = -furpar * (erfst - twrtpi * alphar * expcst) / (rsp * rsq);
    fsr[type - 1] -= furpar * erfst / rsp;
    en0 -= furpar0 * erfst / rsp;
    fpx[ia] += qforce * xab;
    fpy[ia] += qforce * yab;
    fpz[ia] += qforce * zab;
    fpx[ib] -= qforce * xab;
    fpy[ib] -= qforce * yab;
    fpz[ib] -= qforce * zab;
  }
  fs[0] = fsr[0];
  fs[1] = fsr[1];
  *dwrk = fsr[0] + fsr[1] - en0;
}

/* the coupling factors of one 1-4 pair in fnb14_alchemy (src/fnb14_alchemy.f:
 * 149-177 for LJ, 252-289 for the charges): an alchemical atom with
 * lambda 0 counts as normal; one alchemical atom: 1 - |lambda|; two of one
 * lambda: full (and, for the charges, the erf term that restores the full
 * Coulomb the scaled reciprocal sum lacks, 1 - the product of the
 * couplings); two of different lambdas: none (and the reciprocal sum's
 * product subtracted) */
static void alch14_factors(double li, double lj, int charges, double* f, double* f2) {
  *f2 = 0.0;
  if (li == 0.0 && lj != 0.0) {
    *f = 1.0 - fabs(lj);
  } else if (li != 0.0 && lj == 0.0) {
    *f = 1.0 - fabs(li);
  } else if (li == 0.0 && lj == 0.0) {
    *f = 1.0;
  } else if (li != lj) {
    *f = 0.0;
    if (charges) *f2 = -(1.0 - fabs(li)) * (1.0 - fabs(lj));
  } else {
    *f = 1.0;
    if (charges) *f2 = 1.0 - (1.0 - fabs(li)) * (1.0 - fabs(lj));
  }
}

/* fnb14_alchemy, src/fnb14_alchemy.f:225-341 (the Ewald branch): 1-4 pairs
 * with LJ scaled by alch_fact and Coulomb fudge Q_i Q_j [alch_factq erfc/r
 * + alch_factq2 erf/r], at lambda and lambda0 for the work.  ORAC scales
 * only the repulsive term of the LJ force by alch_fact (its energy by
 * alch_fact whole); restated as written.  ue: LJ slt, slv, Coulomb slt,
 * slv; *dwrk: U(lambda) - U(lambda0). */
void orc_fnb14_alchemy(const int* ss_index, const double* xp0, const double* yp0, const double* zp0,
                       const double* charge, const double* ecc12, const double* ecc6, double alphal,
                       const int* int14, int int14p, const int* type14, double fudge, double lj_fudge,
                       const double* lambda, const double* lambdaq, const double* lambda0, const double* lambdaq0,
                       double* fpx, double* fpy, double* fpz, double* ue, double* dwrk) {
  double uconf[2] = {0, 0}, ucoul[2] = {0, 0}, uconf0[2] = {0, 0}, ucoul0[2] = {0, 0};
  double twrtpi = 2.0 / sqrt(PI_D);
  for (int i = 0; i < int14p; i++) {
    int i1 = int14[2 * i] - 1, i2 = int14[2 * i + 1] - 1;
    double af, af0, aq, aq0, aq2, aq20, dum;
    alch14_factors(lambda[i1], lambda[i2], 0, &af, &dum);
    alch14_factors(lambda0[i1], lambda0[i2], 0, &af0, &dum);
    alch14_factors(lambdaq[i1], lambdaq[i2], 1, &aq, &aq2);
    alch14_factors(lambdaq0[i1], lambdaq0[i2], 1, &aq0, &aq20);
    int type = ss_index[i1];
    int lij = type14[i] - 1;
    double xa = xp0[i1] - xp0[i2], ya = yp0[i1] - yp0[i2], za = zp0[i1] - zp0[i2];
    double rsq = xa * xa + ya * ya + za * za;
    double rsp = sqrt(rsq);
    double rsqi = 1.0 / rsq;
    double rspqi = rsqi / rsp;
    double r6 = rsqi * rsqi * rsqi;
    double r12 = r6 * r6;
    double ssvir = af * 12.0 * ecc12[lij] * r12 - 6.0 * ecc6[lij] * r6;
    double qforce = lj_fudge * ssvir * rsqi;
    double aux = lj_fudge * (ecc12[lij] * r12 - ecc6[lij] * r6);
    uconf[type - 1] += af * aux;
    uconf0[type - 1] += af0 * aux;
    double alphar = alphal * rsp;
    double qt = 1.0 / (1.0 + AS_QP * alphar);
    double expcst = exp(-alphar * alphar);
    double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
    double qq = fudge * charge[i1] * charge[i2];
    double furpar = aq * qq, furpar0 = aq0 * qq;
    double erff = 1.0 - erfcst;
    double furpar2 = aq2 * qq, furpar20 = aq20 * qq;
    ucoul[type - 1] += furpar * erfcst / rsp + furpar2 * erff / rsp;
    ucoul0[type - 1] += furpar0 * erfcst / rsp + furpar20 * erff / rsp;
    double a1 = (erfcst + twrtpi * alphar * expcst) * rspqi;
    double a2 = (erff - twrtpi * alphar * expcst) * rspqi;
    qforce += furpar * a1 + furpar2 * a2;
    fpx[i1] += qforce * xa;
    fpy[i1] += qforce * ya;
    fpz[i1] += qforce * za;
    fpx[i2] -= qforce * xa;
    fpy[i2] -= qforce * ya;
    fpz[i2] -= qforce * za;
  }
  ue[0] = uconf[0];
  ue[1] = uconf[1];
  ue[2] = ucoul[0];
  ue[3] = ucoul[1];
  *dwrk = 0.0;
  for (int k = 0; k < 2; k++) *dwrk += uconf[k] + ucoul[k] - (uconf0[k] + ucoul0[k]);
}
