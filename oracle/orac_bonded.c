/*
 * ORACLE — test infrastructure only.
 *
 * FP64 CPU restatement of ORAC's bonded intramolecular forces, the N0/N1
 * terms of mts_intra_n0 / mts_intra_n1: harmonic stretching (fpbond,
 * src/fpbond.f), bending with the Urey-Bradley and stretch-stretch
 * coupling terms (fpbend, src/fpbend.f), proper torsions as Chebyshev
 * polynomials of cos(phi) (fptors, src/fptors.f) and improper torsions
 * (fitors, src/fitors.f).  Coordinates are Cartesian, forces are
 * accumulated, energies are set per solute (ss_index 1) / solvent (2).
 *
 * One deliberate difference: where ORAC meets a torsion with collinear
 * atoms (|sin phi1 sin phi2 sin phi3| < 1e-25) it jitters the four atoms with
 * its random-number generator and retries (src/fptors.f:98-130); here such a
 * term contributes nothing, and orc_fptors returns how many were skipped.
 */
#include <math.h>

#include "orac_oracle.h"

void orc_fpbond(const int* ss_index, const int* lbnd, int nb, const double* x, const double* y, const double* z,
                const double* r0, const double* kb, double* ue, double* fx, double* fy, double* fz) {
  double u[2] = {0.0, 0.0};
  for (int i = 0; i < nb; i++) {
    const int la = lbnd[2 * i] - 1, lb = lbnd[2 * i + 1] - 1;
    const int type = ss_index[la];
    const double x21 = x[lb] - x[la], y21 = y[lb] - y[la], z21 = z[lb] - z[la];
    const double rs21 = sqrt(x21 * x21 + y21 * y21 + z21 * z21);
    const double qforce = -2.0 * kb[i] * (r0[i] - rs21) / rs21;
    fx[la] += qforce * x21;
    fy[la] += qforce * y21;
    fz[la] += qforce * z21;
    fx[lb] -= qforce * x21;
    fy[lb] -= qforce * y21;
    fz[lb] -= qforce * z21;
    u[type - 1] += kb[i] * (rs21 - r0[i]) * (rs21 - r0[i]);
  }
  ue[0] = u[0];
  ue[1] = u[1];
}

/* pot[7*i + k] = pota..potg of bend i: theta0, k, UB r0, UB k, and the
 * coupling parameters (src/fpbend.f:112-178) */
void orc_fpbend(const int* ss_index, const int* lbndg, int nbend, const double* x, const double* y, const double* z,
                const double* pot, double* ue, double* fx, double* fy, double* fz) {
  double u[2] = {0.0, 0.0};
  const double pi = 4.0 * atan(1.0);
  for (int i = 0; i < nbend; i++) {
    const double pota = pot[7 * i], potb = pot[7 * i + 1], potc = pot[7 * i + 2], potd = pot[7 * i + 3];
    const double pote = pot[7 * i + 4], potf = pot[7 * i + 5], potg = pot[7 * i + 6];
    if (fabs(potb) < 1e-12) continue;
    const int la = lbndg[3 * i] - 1, lb = lbndg[3 * i + 1] - 1, lc = lbndg[3 * i + 2] - 1;
    const int type = ss_index[la];
    const double x12 = x[la] - x[lb], y12 = y[la] - y[lb], z12 = z[la] - z[lb];
    const double x32 = x[lc] - x[lb], y32 = y[lc] - y[lb], z32 = z[lc] - z[lb];
    const double rs12 = x12 * x12 + y12 * y12 + z12 * z12;
    const double rs32 = x32 * x32 + y32 * y32 + z32 * z32;
    const double dcc2 = sqrt(rs12 * rs32);
    double cb = (x12 * x32 + y12 * y32 + z12 * z32) / dcc2;
    if (fabs(cb) > 1.0) cb = cb > 0 ? 1.0 : -1.0;
    const double sb = sqrt(1.0 - cb * cb);
    const double bb = acos(cb);
    double qforce;
    if (fabs(pota - pi) < 0.01 || sb < 1e-6)
      qforce = -2.0 * potb;
    else
      qforce = 2.0 * potb * (bb - pota) / sb;
    const double ux1 = x32 / dcc2 - cb * x12 / rs12, ux3 = x12 / dcc2 - cb * x32 / rs32, ux2 = -ux1 - ux3;
    const double uy1 = y32 / dcc2 - cb * y12 / rs12, uy3 = y12 / dcc2 - cb * y32 / rs32, uy2 = -uy1 - uy3;
    const double uz1 = z32 / dcc2 - cb * z12 / rs12, uz3 = z12 / dcc2 - cb * z32 / rs32, uz2 = -uz1 - uz3;
    fx[la] += qforce * ux1;
    fx[lc] += qforce * ux3;
    fx[lb] += qforce * ux2;
    fy[la] += qforce * uy1;
    fy[lc] += qforce * uy3;
    fy[lb] += qforce * uy2;
    fz[la] += qforce * uz1;
    fz[lc] += qforce * uz3;
    fz[lb] += qforce * uz2;
    if (fabs(pota - pi) < 0.01)
      u[type - 1] += 2.0 * potb * (cb + 1.0);
    else
      u[type - 1] += potb * (bb - pota) * (bb - pota);
    /* Urey-Bradley 1-3 spring */
    if (fabs(potd) > 1e-5 && (fabs(pote) < 1e-5 || fabs(potf) > 1e-5)) {
      const double x31 = x[lc] - x[la], y31 = y[lc] - y[la], z31 = z[lc] - z[la];
      const double rsp31 = sqrt(x31 * x31 + y31 * y31 + z31 * z31);
      const double q = -2.0 * potd * (potc - rsp31);
      fx[la] += q * x31 / rsp31;
      fy[la] += q * y31 / rsp31;
      fz[la] += q * z31 / rsp31;
      fx[lc] -= q * x31 / rsp31;
      fy[lc] -= q * y31 / rsp31;
      fz[lc] -= q * z31 / rsp31;
      u[type - 1] += potd * (rsp31 - potc) * (rsp31 - potc);
    }
    /* stretch-stretch coupling */
    int coupling = 0;
    double k12 = 0.0, r1 = 0.0, r2 = 0.0;
    if (fabs(potd) > 1e-5 && fabs(pote) > 1e-5 && fabs(potf) < 1e-5) {
      coupling = 1;
      k12 = potd;
      r1 = potc;
      r2 = pote;
    }
    if (fabs(pote) > 1e-5 && fabs(potf) > 1e-5 && fabs(potg) > 1e-5) {
      coupling = 1;
      k12 = pote;
      r1 = potf;
      r2 = potg;
    }
    if (coupling) {
      const double rsp12 = sqrt(rs12), rsp32 = sqrt(rs32);
      const double qf = k12 * (rsp12 - r1), pf = k12 * (rsp32 - r2);
      const double a1 = x12 / rsp12, b1 = y12 / rsp12, c1 = z12 / rsp12;
      const double a2 = x32 / rsp32, b2 = y32 / rsp32, c2 = z32 / rsp32;
      fx[la] -= pf * a1;
      fy[la] -= pf * b1;
      fz[la] -= pf * c1;
      fx[lb] += pf * a1 + qf * a2;
      fy[lb] += pf * b1 + qf * b2;
      fz[lb] += pf * c1 + qf * c2;
      fx[lc] -= qf * a2;
      fy[lc] -= qf * b2;
      fz[lc] -= qf * c2;
      u[type - 1] += k12 * (rsp12 - r1) * (rsp32 - r2);
    }
  }
  ue[0] = u[0];
  ue[1] = u[1];
}

/* Geometry shared by fptors and fitors: cos(phi) and its gradient with
 * respect to the four atoms (src/fptors.f:69-176).  Returns 0 for a
 * degenerate torsion. */
static int torsion_geom(const double* x, const double* y, const double* z, int l1, int l2, int l3, int l4, int absq,
                        double* coa, double g[4][3], double* sgn) {
  const double x21 = x[l2] - x[l1], y21 = y[l2] - y[l1], z21 = z[l2] - z[l1];
  const double x32 = x[l3] - x[l2], y32 = y[l3] - y[l2], z32 = z[l3] - z[l2];
  const double x43 = x[l4] - x[l3], y43 = y[l4] - y[l3], z43 = z[l4] - z[l3];
  const double rsq21 = x21 * x21 + y21 * y21 + z21 * z21;
  const double rsq32 = x32 * x32 + y32 * y32 + z32 * z32;
  const double rsq43 = x43 * x43 + y43 * y43 + z43 * z43;
  const double rsp21 = sqrt(rsq21), rsp32 = sqrt(rsq32), rsp43 = sqrt(rsq43);
  const double cb1 = (x21 * x32 + y21 * y32 + z21 * z32) / (rsp21 * rsp32);
  const double cb2 = (x43 * x32 + y43 * y32 + z43 * z32) / (rsp43 * rsp32);
  const double cb3 = (x21 * x43 + y21 * y43 + z21 * z43) / (rsp21 * rsp43);
  const double sb1 = sqrt(absq ? fabs(1.0 - cb1 * cb1) : 1.0 - cb1 * cb1);
  const double sb2 = sqrt(absq ? fabs(1.0 - cb2 * cb2) : 1.0 - cb2 * cb2);
  const double sb3 = sqrt(absq ? fabs(1.0 - cb3 * cb3) : 1.0 - cb3 * cb3);
  const double aux = sb1 * sb2;
  if (!(fabs(aux * sb3) >= 1e-25)) return 0;
  double c = (cb1 * cb2 - cb3) / aux;
  if (c > 1.0 && c < 1.000001) c = 1.0;
  if (c < -1.0 && c > -1.000001) c = -1.0;
  double aux1 = cb1 * sb2, aux2 = sb1 * cb2;
  const double auxa = -(aux1 * c + aux2) / aux;
  const double auxb = -(aux2 * c + aux1) / aux;
  const double auxc = sb3 / aux;
  aux1 = rsp21 * rsp32 * sb1;
  aux2 = rsp32 * rsp43 * sb2;
  const double aux3 = rsp21 * rsp43 * sb3;
  const double d[3][3] = {{x21, x32, x43}, {y21, y32, y43}, {z21, z32, z43}};
  for (int k = 0; k < 3; k++) {
    const double v21 = d[k][0], v32 = d[k][1], v43 = d[k][2];
    const double b11 = v32 / aux1 - cb1 * v21 / (rsq21 * sb1);
    const double b13 = -v21 / aux1 + cb1 * v32 / (rsq32 * sb1);
    const double b12 = -b13 - b11;
    const double b22 = v43 / aux2 - cb2 * v32 / (rsq32 * sb2);
    const double b24 = -v32 / aux2 + cb2 * v43 / (rsq43 * sb2);
    const double b23 = -b22 - b24;
    const double b31 = v43 / aux3 - cb3 * v21 / (rsq21 * sb3);
    const double b33 = v21 / aux3 - cb3 * v43 / (rsq43 * sb3);
    const double b32 = -b31, b34 = -b33;
    g[0][k] = auxa * b11 + auxc * b31;
    g[1][k] = auxa * b12 + auxb * b22 + auxc * b32;
    g[2][k] = auxa * b13 + auxb * b23 + auxc * b33;
    g[3][k] = auxb * b24 + auxc * b34;
  }
  *coa = c;
  /* orientation of the dihedral: sign of (r21 x r32) . r43 */
  const double xn = y21 * z32 - y32 * z21, yn = z21 * x32 - z32 * x21, zn = x21 * y32 - x32 * y21;
  *sgn = xn * x43 + yn * y43 + zn * z43;
  return 1;
}

/* cos(n phi) as a polynomial of c = cos(phi), and its derivative (the
 * energy and qforce of src/fptors.f:178-236) */
static int cheb(int n, double c, double* t, double* dt) {
  const double c2 = c * c;
  switch (n) {
    case 1: *t = c; *dt = 1.0; return 1;
    case 2: *t = 2.0 * c2 - 1.0; *dt = 4.0 * c; return 1;
    case 3: *t = 4.0 * c2 * c - 3.0 * c; *dt = 12.0 * c2 - 3.0; return 1;
    case 4: *t = 8.0 * c2 * c2 - 8.0 * c2 + 1.0; *dt = 32.0 * c2 * c - 16.0 * c; return 1;
    case 5:
      *t = 16.0 * c2 * c2 * c - 20.0 * c2 * c + 5.0 * c;
      *dt = 80.0 * c2 * c2 - 60.0 * c2 + 5.0;
      return 1;
    case 6:
      *t = 32.0 * c2 * c2 * c2 - 48.0 * c2 * c2 + 18.0 * c2 - 1.0;
      *dt = 192.0 * c2 * c2 * c - 192.0 * c2 * c + 36.0 * c;
      return 1;
    case 7:
      *t = 64.0 * c2 * c2 * c2 * c - 112.0 * c2 * c2 * c + 56.0 * c2 * c - 7.0 * c;
      *dt = 448.0 * c2 * c2 * c2 - 560.0 * c2 * c2 + 168.0 * c2 - 7.0;
      return 1;
    case 8:
      *t = 128.0 * c2 * c2 * c2 * c2 - 256.0 * c2 * c2 * c2 + 160.0 * c2 * c2 - 32.0 * c2 + 1.0;
      *dt = 1024.0 * c2 * c2 * c2 * c - 1536.0 * c2 * c2 * c + 640.0 * c2 * c - 64.0 * c;
      return 1;
    default: return 0;
  }
}

/* fptors: pota = +-n (sign: phase 0 or pi), potb = V:
 * U = sig (|V| - V cos(n phi)).  Multiplicities 1..8; ORAC's two special
 * forms (12, 14) are not restated and count as skipped.  Returns the number
 * of terms skipped (degenerate or unsupported). */
int orc_fptors(const int* ss_index, const int* ltor, int nt, const double* x, const double* y, const double* z,
               const double* pota, const double* potb, double* ue, double* fx, double* fy, double* fz) {
  double u[2] = {0.0, 0.0};
  int skipped = 0;
  for (int i = 0; i < nt; i++) {
    if (fabs(potb[i]) < 1e-12) continue;
    const int l1 = ltor[4 * i] - 1, l2 = ltor[4 * i + 1] - 1, l3 = ltor[4 * i + 2] - 1, l4 = ltor[4 * i + 3] - 1;
    const int tmp = (int)lround(pota[i]);
    const int ntph = tmp < 0 ? -tmp : tmp;
    const double sig = tmp < 0 ? -1.0 : 1.0;
    double coa, g[4][3], sgn, t, dt;
    if (ntph < 1 || !cheb(ntph, 0.5, &t, &dt) ||
        !torsion_geom(x, y, z, l1, l2, l3, l4, 1, &coa, g, &sgn)) {
      skipped++;
      continue;
    }
    cheb(ntph, coa, &t, &dt);
    const double enrg = sig * (fabs(potb[i]) - t * potb[i]);
    const double qforce = sig * dt * potb[i];
    u[ss_index[l1] - 1] += enrg;
    const int l[4] = {l1, l2, l3, l4};
    for (int a = 0; a < 4; a++) {
      fx[l[a]] += qforce * g[a][0];
      fy[l[a]] += qforce * g[a][1];
      fz[l[a]] += qforce * g[a][2];
    }
  }
  ue[0] = u[0];
  ue[1] = u[1];
  return skipped;
}

/* fitors: potc > 0 harmonic in the dihedral angle, U = V (phi - phi0)^2
 * with ORAC's branch choices for phi (src/fitors.f:178-201); otherwise the
 * cosine form of fptors with pota = +-n.  Returns the number skipped. */
int orc_fitors(const int* ss_index, const int* litr, int nt, const double* x, const double* y, const double* z,
               const double* pota, const double* potb, const double* potc, double* ue, double* fx, double* fy,
               double* fz) {
  double u[2] = {0.0, 0.0};
  int skipped = 0;
  for (int i = 0; i < nt; i++) {
    if (fabs(potb[i]) < 1e-12) continue;
    const int l1 = litr[4 * i] - 1, l2 = litr[4 * i + 1] - 1, l3 = litr[4 * i + 2] - 1, l4 = litr[4 * i + 3] - 1;
    double coa, g[4][3], sgn;
    if (!torsion_geom(x, y, z, l1, l2, l3, l4, 0, &coa, g, &sgn)) {
      skipped++;
      continue;
    }
    double enrg, qforce;
    if (potc[i] > 0.0) {
      double bb = acos(coa);
      const double aux4 = sgn >= 0 ? bb : -bb; /* Fortran SIGN(bb, s) */
      if (aux4 < 0.0 && fabs(aux4) >= 1.57079) {
        bb = 2.0 * acos(-1.0) + aux4;
        if (fabs(pota[i] - bb) > 3.14159) bb = -2 * 3.14159 + bb;
      } else if (aux4 < 0.0 && fabs(aux4) < 1.57079) {
        bb = aux4;
        if (fabs(pota[i] - bb) > 3.14159) bb = 2 * 3.14159 + bb;
      } else {
        bb = aux4;
        if (fabs(pota[i] - bb) > 3.14159) bb = 2 * 3.14159 + bb;
        if (fabs(pota[i] - bb) > 3.14159) bb = -4 * 3.14159 + bb;
      }
      if (fabs(pota[i]) < 1e-3)
        qforce = 2.0 * potb[i];
      else if (fabs(pota[i] - 3.14159) < 1e-3)
        qforce = -2.0 * potb[i];
      else
        qforce = 2.0 * potb[i] * (bb - pota[i]) / sin(bb);
      enrg = potb[i] * (bb - pota[i]) * (bb - pota[i]);
    } else {
      const int tmp = (int)lround(pota[i]);
      const int ntph = tmp < 0 ? -tmp : tmp;
      const double sig = tmp < 0 ? -1.0 : 1.0;
      double t, dt;
      if (ntph < 1 || !cheb(ntph, coa, &t, &dt)) {
        skipped++;
        continue;
      }
      enrg = sig * (fabs(potb[i]) - t * potb[i]);
      qforce = sig * dt * potb[i];
    }
    u[ss_index[l1] - 1] += enrg;
    const int l[4] = {l1, l2, l3, l4};
    for (int a = 0; a < 4; a++) {
      fx[l[a]] += qforce * g[a][0];
      fy[l[a]] += qforce * g[a][1];
      fz[l[a]] += qforce * g[a][2];
    }
  }
  ue[0] = u[0];
  ue[1] = u[1];
  return skipped;
}
