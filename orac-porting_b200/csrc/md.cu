// r-RESPA molecular dynamics driver on the device: the NVE part of ORAC's
// mtsmd step loop (src/mtsmd.f:2390-3540) with its kick/drift routines
// correc (src/correc.f), verlet (src/verlet.f) and the SHAKE/RATTLE
// constraint solvers (src/rattle_verlet.f, src/rattle_correc.f).
//
// State lives in HBM: FP64 positions and velocities, and one int64
// fixed-point force accumulator per RESPA level (H, L, M) that the shell
// kernels and the SPME gather add into and the kicks read.  One outer (H)
// step:
//
//   [every nupdte steps] linked-cell H list, phony 'h' (L list), phony 'l'
//                        (M list)                       src/mtsmd.f:2403-2470
//   H half kick + RATTLE                                        :2477-2484
//   do lrespa:   L half kick + RATTLE
//     do mrespa: M half kick + RATTLE
//                drift (verlet) + SHAKE + RATTLE, scaled frame, group
//                centres, pair-kernel inputs      (one fused kernel)
//                M shell forces                                    :3030
//                M half kick + RATTLE
//     L shell forces (+ SPME when the reciprocal shell is L)   :3185-3201
//     L half kick + RATTLE
//   H shell forces (+ SPME when the reciprocal shell is H)     :3263-3278
//   phony 'l' refresh of the M list                            :3287-3295
//   H half kick + RATTLE
//
// Constraints.  Molecules with at most 3 constraints on at most 4 atoms (the
// rigid waters) are solved by one thread with the molecule in registers, as
// ORAC's matrix-inversion branch does for small molecules
// (src/rattle_verlet.f:228-330): Newton iterations on the linearised
// constraint system for SHAKE (converged to 1e-12 A^2, well inside ORAC's
// 1e-8) and one exact linear solve for the RATTLE velocity step.  Larger
// constrained molecules use the iterative branch (tolerance 1e-8 A^2, 5000
// iterations, src/rattle_verlet.f:76,209).
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace {

constexpr int SMA = 4;  // atoms of a register-solved molecule
constexpr int SMC = 3;  // constraints of a register-solved molecule
constexpr int NLV = 5;  // r-RESPA force levels: H, L, M, N1, N0
enum { LH = 0, LL = 1, LM = 2, LN1 = 3, LN0 = 4 };

__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// Gaussian elimination without pivoting for n <= 3 (the matrices are
// J M^-1 J^T products: symmetric positive definite up to the small
// difference between old and new bond vectors).  Returns false on a zero
// pivot.
__device__ __forceinline__ bool solve3(double A[SMC][SMC], double b[SMC], int n) {
#pragma unroll
  for (int k = 0; k < SMC; k++) {
    if (k < n) {
      if (A[k][k] == 0.0) return false;
      const double inv = 1.0 / A[k][k];
#pragma unroll
      for (int i = k + 1; i < SMC; i++) {
        if (i < n) {
          const double f = A[i][k] * inv;
#pragma unroll
          for (int j = k; j < SMC; j++) A[i][j] -= f * A[k][j];
          b[i] -= f * b[k];
        }
      }
    }
  }
#pragma unroll
  for (int k = SMC - 1; k >= 0; k--) {
    if (k < n) {
      double s = b[k];
#pragma unroll
      for (int j = k + 1; j < SMC; j++)
        if (j < n) s -= A[k][j] * b[j];
      b[k] = s / A[k][k];
    }
  }
  return true;
}

struct ThermoDev {
  double eta[3], etap[3], s[3];  // s = exp(-tm/4 etap): the scales of the sandwiches
  double q[3], ndfkt[3];
  double tm, tm4;
  unsigned int count;  // blocks of the pass done; the last one updates the thermostats
};

// sums per molecule outside the small molecules (k_mol_sums): m v, then the
// forces of the levels N0, N1, M, L, H (sum of f), all in the fixed point of
// the force accumulators (integer sums: exact, the same in any order)
constexpr int TH_NS = 18;

// the M half kick cm of force f (mass 1/im) between the two scalings of a
// thermostat sandwich: the velocity relative to the molecule's centre of
// mass (V; M force F, mass 1/iM) by sk, the centre of mass by sc
__device__ __forceinline__ double sandwich(double v, double f, double im, double V, double F, double iM, double sk,
                                           double sc, double cm) {
  return sk * (sk * (v - V) + cm * (f * im - F * iM)) + sc * (sc * V + cm * F * iM);
}

struct MolArgs {
  int N;
  // small constrained molecules
  int nsm;
  const int4* sm;      // (first atom, natoms, first constraint, nconstraints)
  const int2* smg;     // (first group, ngroups)
  const int2* cloc;    // constraint atoms, local to the molecule
  const double* dss;   // squared lengths
  // atoms handled one by one (everything outside small molecules)
  int nfree;
  const int* free_atoms;
  int nfreeg;
  const int* free_groups;
  // the drift's split of the free atoms: groups of unconstrained molecules
  // (one thread drifts the group's atoms and sets its centre) and atoms of
  // large constrained molecules (one thread each; their groups follow the
  // iterative SHAKE in k_free_groups)
  int ndg;
  const int* drift_groups;
  int nda;
  const int* drift_atoms;
  const int* sm_atoms;  // atoms of the constraint clusters
  // state
  double* x;
  double* xo;
  double* v;
  const double* invm;
  const double* pm;
  const float* q;
  const int2* gmeta;
  // scaled frame and pair-kernel inputs
  double o11, o12, o13, o22, o23, o33;
  double c11, c12, c13, c22, c23, c33;
  int G;
  double* grp;       // [3G] scaled group centres (for the list builder)
  double4* gpos;     // [G]
  float4* aoff;      // [N]
  // kick: v += sum_l ck[l] f_l / m over the level accumulators, then RATTLE
  // (several correc + rattle_correc calls of one instant merged: RATTLE is a
  // linear projection, so one projection of the summed kick is the same)
  const unsigned long long* fk[NLV];
  double ck[NLV];
  int kick;
  // the N0 force of the verlet step (src/verlet.f: half kick without
  // RATTLE, then the drift), or null
  const unsigned long long* fv;
  // accumulators zeroed for the evaluations that follow this drift
  unsigned long long* fz[NLV];
  double dt;
  double idt;  // 1 / dt, 0 for a zero step
  int groups;  // group centres and pair-kernel inputs wanted (a shell evaluation follows)
  double tol;
  int* flag;
  // the start sandwich of an M step under thermostats (k_drift<true>): the
  // thermostats' scales, each atom's thermostat (1 solute, 2 solvent) and
  // molecule outside the small ones, those molecules' centre-of-mass
  // velocities, sums and masses, tm/2
  const ThermoDev* th;
  const int* tcls;
  const int* abm;
  const double* vcur;
  const unsigned long long* msum;
  const double* bmass;
  double tcm;
};

// a constraint cluster of a large molecule (the atoms joined by one
// connected set of constraints, at most SMA atoms and SMC constraints):
// solved like a small molecule, its atoms listed in sm_atoms from m.x, no
// groups of its own (the molecule's groups are centred after every atom
// of the molecule has moved)
constexpr int CLUSTER = 1024;

// atom a of small molecule or constraint cluster m
__device__ __forceinline__ int sm_atom(const MolArgs& A, const int4& m, int a) {
  return (m.w & CLUSTER) ? A.sm_atoms[m.x + a] : m.x + a;
}


__device__ __forceinline__ double fixd(unsigned long long v) { return (double)(long long)v * ORAC_FSCALE_INV; }

// RATTLE velocity projection of one small molecule held in registers
__device__ __forceinline__ bool rattle_small(double x[SMA][3], double v[SMA][3], const double im[SMA], const int2* c,
                                             int nc) {
  double r[SMC][3], M[SMC][SMC], rhs[SMC];
  int ca[SMC], cb[SMC];
#pragma unroll
  for (int k = 0; k < SMC; k++) {
    if (k < nc) {
      ca[k] = c[k].x;
      cb[k] = c[k].y;
    } else {
      ca[k] = cb[k] = 0;
    }
  }
#pragma unroll
  for (int k = 0; k < SMC; k++) {
    if (k < nc) {
      double va[3], vb[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        double xa = 0, xb = 0;
#pragma unroll
        for (int a = 0; a < SMA; a++) {
          if (a == ca[k]) {
            xa = x[a][d];
            va[d] = v[a][d];
          }
          if (a == cb[k]) {
            xb = x[a][d];
            vb[d] = v[a][d];
          }
        }
        r[k][d] = xa - xb;
      }
      rhs[k] = -(r[k][0] * (va[0] - vb[0]) + r[k][1] * (va[1] - vb[1]) + r[k][2] * (va[2] - vb[2]));
    }
  }
#pragma unroll
  for (int k = 0; k < SMC; k++)
#pragma unroll
    for (int l = 0; l < SMC; l++) {
      if (k < nc && l < nc) {
        double ia = 0, ib = 0;
#pragma unroll
        for (int a = 0; a < SMA; a++) {
          if (a == ca[k]) ia = im[a];
          if (a == cb[k]) ib = im[a];
        }
        const double cc = (ca[k] == ca[l] ? ia : 0.0) - (ca[k] == cb[l] ? ia : 0.0) - (cb[k] == ca[l] ? ib : 0.0) +
                          (cb[k] == cb[l] ? ib : 0.0);
        M[k][l] = cc * dot3(r[k], r[l]);
      } else {
        M[k][l] = 0.0;
      }
    }
  if (!solve3(M, rhs, nc)) return false;
#pragma unroll
  for (int l = 0; l < SMC; l++) {
    if (l < nc) {
#pragma unroll
      for (int a = 0; a < SMA; a++) {
        const double s = (a == ca[l]) ? 1.0 : ((a == cb[l]) ? -1.0 : 0.0);
        if (s != 0.0) {
          v[a][0] += s * rhs[l] * r[l][0] * im[a];
          v[a][1] += s * rhs[l] * r[l][1] * im[a];
          v[a][2] += s * rhs[l] * r[l][2] * im[a];
        }
      }
    }
  }
  return true;
}

// SHAKE of one small molecule: Newton iterations on g_k = |d_k|^2 - L_k^2
// with displacements along the old bond vectors r0_l, positions and
// velocities corrected in place.
__device__ __forceinline__ bool shake_small(double x[SMA][3], const double xo[SMA][3], double v[SMA][3],
                                            const double im[SMA], const int2* c, const double* L2, int nc, double dt,
                                            double tol) {
  int ca[SMC], cb[SMC];
  double r0[SMC][3], lam[SMC];
#pragma unroll
  for (int k = 0; k < SMC; k++) {
    lam[k] = 0.0;
    if (k < nc) {
      ca[k] = c[k].x;
      cb[k] = c[k].y;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        double xa = 0, xb = 0;
#pragma unroll
        for (int a = 0; a < SMA; a++) {
          if (a == ca[k]) xa = xo[a][d];
          if (a == cb[k]) xb = xo[a][d];
        }
        r0[k][d] = xa - xb;
      }
    } else {
      ca[k] = cb[k] = 0;
      r0[k][0] = r0[k][1] = r0[k][2] = 0.0;
    }
  }
  bool ok = false;
  for (int it = 0; it < 50; it++) {
    double dk[SMC][3], g[SMC];
    double gmax = 0.0;
#pragma unroll
    for (int k = 0; k < SMC; k++) {
      if (k < nc) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
          double xa = 0, xb = 0;
#pragma unroll
          for (int a = 0; a < SMA; a++) {
            if (a == ca[k]) xa = x[a][d];
            if (a == cb[k]) xb = x[a][d];
          }
          dk[k][d] = xa - xb;
        }
        g[k] = -(dot3(dk[k], dk[k]) - L2[k]);
        gmax = fmax(gmax, fabs(g[k]));
      } else {
        g[k] = 0.0;
      }
    }
    if (gmax < tol) {
      ok = true;
      break;
    }
    double J[SMC][SMC];
#pragma unroll
    for (int k = 0; k < SMC; k++)
#pragma unroll
      for (int l = 0; l < SMC; l++) {
        if (k < nc && l < nc) {
          double ia = 0, ib = 0;
#pragma unroll
          for (int a = 0; a < SMA; a++) {
            if (a == ca[k]) ia = im[a];
            if (a == cb[k]) ib = im[a];
          }
          const double cc = (ca[k] == ca[l] ? ia : 0.0) - (ca[k] == cb[l] ? ia : 0.0) -
                            (cb[k] == ca[l] ? ib : 0.0) + (cb[k] == cb[l] ? ib : 0.0);
          J[k][l] = 2.0 * cc * dot3(dk[k], r0[l]);
        } else {
          J[k][l] = 0.0;
        }
      }
    if (!solve3(J, g, nc)) return false;
#pragma unroll
    for (int l = 0; l < SMC; l++) {
      if (l < nc) {
        lam[l] += g[l];
#pragma unroll
        for (int a = 0; a < SMA; a++) {
          const double s = (a == ca[l]) ? 1.0 : ((a == cb[l]) ? -1.0 : 0.0);
          if (s != 0.0) {
            x[a][0] += s * g[l] * r0[l][0] * im[a];
            x[a][1] += s * g[l] * r0[l][1] * im[a];
            x[a][2] += s * g[l] * r0[l][2] * im[a];
          }
        }
      }
    }
  }
  if (dt != 0.0) {
    const double dti = 1.0 / dt;
#pragma unroll
    for (int l = 0; l < SMC; l++) {
      if (l < nc) {
#pragma unroll
        for (int a = 0; a < SMA; a++) {
          const double s = (a == ca[l]) ? 1.0 : ((a == cb[l]) ? -1.0 : 0.0);
          if (s != 0.0) {
            v[a][0] += s * lam[l] * r0[l][0] * im[a] * dti;
            v[a][1] += s * lam[l] * r0[l][1] * im[a] * dti;
            v[a][2] += s * lam[l] * r0[l][2] * im[a] * dti;
          }
        }
      }
    }
  }
  return ok;
}

// Star clusters: a centre atom (local 0) bonded by constraint k to atom k+1
// (a heavy atom with its hydrogens).  The same Newton SHAKE and exact
// RATTLE as shake_small / rattle_small with the topology known at compile
// time: J_kl = 2 (im_0 + [k == l] im_{k+1}) d_k . r0_l.
template <int NC>
__device__ __forceinline__ bool solve_n(double A[NC][NC], double b[NC]) {
#pragma unroll
  for (int k = 0; k < NC; k++) {
    if (A[k][k] == 0.0) return false;
    const double inv = 1.0 / A[k][k];
#pragma unroll
    for (int i = k + 1; i < NC; i++) {
      const double f = A[i][k] * inv;
#pragma unroll
      for (int j = k; j < NC; j++) A[i][j] -= f * A[k][j];
      b[i] -= f * b[k];
    }
  }
#pragma unroll
  for (int k = NC - 1; k >= 0; k--) {
    double t = b[k];
#pragma unroll
    for (int j = k + 1; j < NC; j++) t -= A[k][j] * b[j];
    b[k] = t / A[k][k];
  }
  return true;
}

template <int NC>
__device__ __forceinline__ bool shake_star(double x[SMA][3], const double xo[SMA][3], double v[SMA][3],
                                           const double im[SMA], const double* L2, double idt, double tol) {
  double r0[NC][3], lam[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) {
    lam[k] = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) r0[k][d] = xo[0][d] - xo[k + 1][d];
  }
  bool ok = false;
  for (int it = 0; it < 50; it++) {
    double dk[NC][3], g[NC], gmax = 0.0;
#pragma unroll
    for (int k = 0; k < NC; k++) {
#pragma unroll
      for (int d = 0; d < 3; d++) dk[k][d] = x[0][d] - x[k + 1][d];
      g[k] = -(dot3(dk[k], dk[k]) - L2[k]);
      gmax = fmax(gmax, fabs(g[k]));
    }
    if (gmax < tol) {
      ok = true;
      break;
    }
    double J[NC][NC];
#pragma unroll
    for (int k = 0; k < NC; k++)
#pragma unroll
      for (int l = 0; l < NC; l++) J[k][l] = 2.0 * (im[0] + (k == l ? im[k + 1] : 0.0)) * dot3(dk[k], r0[l]);
    if (!solve_n<NC>(J, g)) return false;
#pragma unroll
    for (int l = 0; l < NC; l++) {
      lam[l] += g[l];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        x[0][d] += g[l] * r0[l][d] * im[0];
        x[l + 1][d] -= g[l] * r0[l][d] * im[l + 1];
      }
    }
  }
#pragma unroll
  for (int l = 0; l < NC; l++)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      v[0][d] += lam[l] * r0[l][d] * im[0] * idt;
      v[l + 1][d] -= lam[l] * r0[l][d] * im[l + 1] * idt;
    }
  return ok;
}

template <int NC>
__device__ __forceinline__ bool rattle_star(const double x[SMA][3], double v[SMA][3], const double im[SMA]) {
  double r[NC][3], rhs[NC], M[NC][NC];
#pragma unroll
  for (int k = 0; k < NC; k++) {
#pragma unroll
    for (int d = 0; d < 3; d++) r[k][d] = x[0][d] - x[k + 1][d];
    rhs[k] = -(r[k][0] * (v[0][0] - v[k + 1][0]) + r[k][1] * (v[0][1] - v[k + 1][1]) +
               r[k][2] * (v[0][2] - v[k + 1][2]));
  }
#pragma unroll
  for (int k = 0; k < NC; k++)
#pragma unroll
    for (int l = 0; l < NC; l++) M[k][l] = (im[0] + (k == l ? im[k + 1] : 0.0)) * dot3(r[k], r[l]);
  if (!solve_n<NC>(M, rhs)) return false;
#pragma unroll
  for (int l = 0; l < NC; l++)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      v[0][d] += rhs[l] * r[l][d] * im[0];
      v[l + 1][d] -= rhs[l] * r[l][d] * im[l + 1];
    }
  return true;
}

__device__ __forceinline__ bool rattle_star_n(int nc, const double x[SMA][3], double v[SMA][3],
                                              const double im[SMA]) {
  return nc == 1 ? rattle_star<1>(x, v, im) : (nc == 2 ? rattle_star<2>(x, v, im) : rattle_star<3>(x, v, im));
}

__device__ __forceinline__ bool shake_star_n(int nc, double x[SMA][3], const double xo[SMA][3], double v[SMA][3],
                                             const double im[SMA], const double* L2, double idt, double tol) {
  return nc == 1 ? shake_star<1>(x, xo, v, im, L2, idt, tol)
                 : (nc == 2 ? shake_star<2>(x, xo, v, im, L2, idt, tol) : shake_star<3>(x, xo, v, im, L2, idt, tol));
}

// Rigid three-atom molecules (the waters) with constraints (0,1), (0,2),
// (1,2) in this order: the same Newton SHAKE and exact RATTLE as above with
// the constraint topology fixed at compile time and the 3x3 systems solved
// in closed form (adjugate over determinant).  MOL3 in the molecule record
// marks them.
constexpr int MOL3 = 256;
// a small molecule none of whose atoms has an intramolecular-level term
constexpr int NOINTRA = 512;
// a star cluster (shake_star / rattle_star): centre first, constraints (0, k+1)
constexpr int STAR = 2048;

__device__ __forceinline__ bool solve3x3(const double J[3][3], const double g[3], double out[3]) {
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  if (det == 0.0 || !isfinite(det)) return false;
  const double id = 1.0 / det;
  const double c10 = J[0][2] * J[2][1] - J[0][1] * J[2][2];
  const double c11 = J[0][0] * J[2][2] - J[0][2] * J[2][0];
  const double c12 = J[0][1] * J[2][0] - J[0][0] * J[2][1];
  const double c20 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  const double c21 = J[0][2] * J[1][0] - J[0][0] * J[1][2];
  const double c22 = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  out[0] = (c00 * g[0] + c10 * g[1] + c20 * g[2]) * id;
  out[1] = (c01 * g[0] + c11 * g[1] + c21 * g[2]) * id;
  out[2] = (c02 * g[0] + c12 * g[1] + c22 * g[2]) * id;
  return true;
}

// coupling of constraints k = (a,b), l = (c,d) through the shared atoms:
// delta(a,c) im_a - delta(a,d) im_a - delta(b,c) im_b + delta(b,d) im_b
__device__ __forceinline__ void coupling3(const double im[SMA], double cc[3][3]) {
  cc[0][0] = im[0] + im[1];
  cc[0][1] = im[0];
  cc[0][2] = -im[1];
  cc[1][0] = im[0];
  cc[1][1] = im[0] + im[2];
  cc[1][2] = im[2];
  cc[2][0] = -im[1];
  cc[2][1] = im[2];
  cc[2][2] = im[1] + im[2];
}

__device__ __forceinline__ void bonds3(const double x[SMA][3], double r[3][3]) {
#pragma unroll
  for (int d = 0; d < 3; d++) {
    r[0][d] = x[0][d] - x[1][d];
    r[1][d] = x[0][d] - x[2][d];
    r[2][d] = x[1][d] - x[2][d];
  }
}

// add lambda_l * r_l * im to atom a and subtract it from atom b of each constraint
__device__ __forceinline__ void apply3(double y[SMA][3], const double lam[3], const double r[3][3], const double im[SMA],
                                       double scale) {
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double u0 = lam[0] * r[0][d] * scale, u1 = lam[1] * r[1][d] * scale, u2 = lam[2] * r[2][d] * scale;
    y[0][d] += (u0 + u1) * im[0];
    y[1][d] += (u2 - u0) * im[1];
    y[2][d] -= (u1 + u2) * im[2];
  }
}

__device__ __forceinline__ bool rattle3(const double x[SMA][3], double v[SMA][3], const double im[SMA]) {
  double r[3][3], cc[3][3], M[3][3], rhs[3], lam[3];
  bonds3(x, r);
  coupling3(im, cc);
  const int ca[3] = {0, 0, 1}, cb[3] = {1, 2, 2};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    rhs[k] = -(r[k][0] * (v[ca[k]][0] - v[cb[k]][0]) + r[k][1] * (v[ca[k]][1] - v[cb[k]][1]) +
               r[k][2] * (v[ca[k]][2] - v[cb[k]][2]));
#pragma unroll
    for (int l = 0; l < 3; l++) M[k][l] = cc[k][l] * dot3(r[k], r[l]);
  }
  if (!solve3x3(M, rhs, lam)) return false;
  apply3(v, lam, r, im, 1.0);
  return true;
}

__device__ __forceinline__ bool shake3(double x[SMA][3], const double xo[SMA][3], double v[SMA][3],
                                       const double im[SMA], const double* L2, double dt, double tol) {
  double r0[3][3], cc[3][3], lam[3] = {0.0, 0.0, 0.0};
  bonds3(xo, r0);
  coupling3(im, cc);
  bool ok = false;
  for (int it = 0; it < 50; it++) {
    double dk[3][3], g[3], J[3][3], dl[3];
    bonds3(x, dk);
    double gmax = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      g[k] = -(dot3(dk[k], dk[k]) - L2[k]);
      gmax = fmax(gmax, fabs(g[k]));
    }
    if (gmax < tol) {
      ok = true;
      break;
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) J[k][l] = 2.0 * cc[k][l] * dot3(dk[k], r0[l]);
    if (!solve3x3(J, g, dl)) return false;
#pragma unroll
    for (int l = 0; l < 3; l++) lam[l] += dl[l];
    apply3(x, dl, r0, im, 1.0);
  }
  if (dt != 0.0) apply3(v, lam, r0, im, 1.0 / dt);
  return ok;
}

// SETTLE (Miyamoto and Kollman, J. Comput. Chem. 13, 952 (1992)): the SHAKE
// solution for a rigid isosceles triangle (atom 0 the apex, equal masses
// and lengths to atoms 1 and 2) in closed form.  The constraint forces lie
// along the old bonds, so in the frame whose z axis is the old plane's
// normal the z coordinates keep their unconstrained values; they fix the
// two tilts of the canonical triangle (phi about x, psi about y), and the
// turn theta about z follows from the zero torque of forces along the old
// bonds: sum_i m_i (x0_i dy_i - y0_i dx_i) = 0 with d = constrained -
// unconstrained, i.e. alpha sin(theta) + beta cos(theta) = gamma.  x holds
// the unconstrained positions on entry, the constrained ones on exit; v
// gains the displacement / dt.  Returns false where no solution exists.
__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ bool settle3(double x[SMA][3], const double xo[SMA][3], double v[SMA][3], const double im[SMA],
                        const double* L2, double idt) {
  // mass fractions from the inverse masses: mA / (mA + 2 mB) = imB / (imB + 2 imA)
  const double iM = 1.0 / (im[1] + 2.0 * im[0]);
  const double wA = im[1] * iM, wB = im[0] * iM;
  const double rc = 0.5 * sqrt(L2[2]);
  const double h2 = L2[0] - rc * rc;
  if (!(h2 > 0.0)) return false;
  const double h = sqrt(h2), ra = 2.0 * wB * h, rb = wA * h;  // apex and base from the centre of mass
  double d[3], a1[3], b1[3], c1[3], b0[3], c0[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    d[k] = wA * x[0][k] + wB * (x[1][k] + x[2][k]);
    a1[k] = x[0][k] - d[k];
    b1[k] = x[1][k] - d[k];
    c1[k] = x[2][k] - d[k];
    b0[k] = xo[1][k] - xo[0][k];
    c0[k] = xo[2][k] - xo[0][k];
  }
  double ez[3], ex[3], ey[3];
  cross3(b0, c0, ez);
  cross3(a1, ez, ex);
  cross3(ez, ex, ey);
  const double nz = dot3(ez, ez), nx = dot3(ex, ex), ny = dot3(ey, ey);
  if (!(nz > 0.0 && nx > 0.0 && ny > 0.0)) return false;
  const double iz = rsqrt(nz), ix = rsqrt(nx), iy = rsqrt(ny);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    ez[k] *= iz;
    ex[k] *= ix;
    ey[k] *= iy;
  }
  const double b0x = dot3(ex, b0), b0y = dot3(ey, b0), c0x = dot3(ex, c0), c0y = dot3(ey, c0);
  const double a1z = dot3(ez, a1);
  const double b1x = dot3(ex, b1), b1y = dot3(ey, b1), b1z = dot3(ez, b1);
  const double c1x = dot3(ex, c1), c1y = dot3(ey, c1), c1z = dot3(ez, c1);
  const double sphi = a1z / ra;
  if (!(fabs(sphi) < 1.0)) return false;
  const double cphi = sqrt(1.0 - sphi * sphi);
  const double spsi = (b1z - c1z) / (2.0 * rc * cphi);
  if (!(fabs(spsi) < 1.0)) return false;
  const double cpsi = sqrt(1.0 - spsi * spsi);
  // the canonical triangle tilted by phi and psi
  const double a2y = ra * cphi, a2z = ra * sphi;
  const double b2x = -rc * cpsi, b2y = -rb * cphi - rc * spsi * sphi, b2z = -rb * sphi + rc * spsi * cphi;
  const double c2x = rc * cpsi, c2y = -rb * cphi + rc * spsi * sphi, c2z = -rb * sphi - rc * spsi * cphi;
  // the turn about z (the apex term vanishes: its old position is the origin)
  const double alpha = b0x * b2x + b0y * b2y + c0x * c2x + c0y * c2y;
  const double beta = b0x * b2y - b0y * b2x + c0x * c2y - c0y * c2x;
  const double gamma = b0x * b1y - b0y * b1x + c0x * c1y - c0y * c1x;
  const double ab2 = alpha * alpha + beta * beta, disc = ab2 - gamma * gamma;
  if (!(disc >= 0.0 && ab2 > 0.0)) return false;
  const double sth = (alpha * gamma - beta * sqrt(disc)) / ab2;
  const double cth = sqrt(1.0 - sth * sth);
  const double p[3][3] = {{-a2y * sth, a2y * cth, a2z},
                          {b2x * cth - b2y * sth, b2x * sth + b2y * cth, b2z},
                          {c2x * cth - c2y * sth, c2x * sth + c2y * cth, c2z}};
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double xn = d[k] + ex[k] * p[a][0] + ey[k] * p[a][1] + ez[k] * p[a][2];
      v[a][k] += (xn - x[a][k]) * idt;
      x[a][k] = xn;
    }
  return true;
}

// levels 0..nlev-1 (molecules without intramolecular terms have nothing at
// the N1 and N0 levels: nlev = 3)
__device__ __forceinline__ double kick_dv(const MolArgs& A, int i, int nlev = NLV) {
  double dv = 0.0;
#pragma unroll
  for (int l = 0; l < NLV; l++)
    if (l < nlev && A.ck[l] != 0.0) dv += A.ck[l] * fixd(A.fk[l][i]);
  return dv;
}

// free atom i (SoA component index d*N + g): kick, verlet half kick of the N0
// force and drift, zeroing of the level accumulators that restart here
template <bool TH>
__device__ __forceinline__ void drift_atom(const MolArgs& A, int g, double dt) {
  const int N = A.N;
  const double im = A.invm[g];
  int p = 0;
  double sc = 1.0, sk = 1.0, iM = 0.0;
  if constexpr (TH) {
    p = A.abm[g];
    sc = A.th->s[0];
    sk = A.th->s[A.tcls[g]];
    iM = 1.0 / A.bmass[p];
  }
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int i = d * N + g;
    const double f = A.fv ? fixd(A.fv[i]) : 0.0;
    double v = A.v[i];
    if constexpr (TH)
      v = sandwich(v, fixd(A.fk[LM][i]), im, A.vcur[3 * p + d], fixd(A.msum[(size_t)p * TH_NS + 9 + d]), iM, sk, sc,
                   A.tcm);
    if (A.kick) v += kick_dv(A, i) * im;
    const double xo = A.x[i];
    A.xo[i] = xo;
    A.x[i] = xo + dt * v + f * 0.5 * dt * dt * im;
    A.v[i] = v + f * 0.5 * dt * im;
#pragma unroll
    for (int l = 0; l < NLV; l++)
      if (A.fz[l]) A.fz[l][i] = 0ull;
  }
}

// scaled centre of group gi from its atoms' positions and the pair-kernel
// inputs of its atoms (appbou, src/appbou.f:57-69)
__device__ __forceinline__ void group_centre(const MolArgs& A, int gi) {
  const int N = A.N;
  const int2 mg = A.gmeta[gi];
  const int a0 = mg.x, n = mg.y & 0xff;
  double c[3] = {0, 0, 0};
  for (int a = a0; a < a0 + n; a++) {
    const double x = A.x[a], y = A.x[N + a], z = A.x[2 * N + a];
    const double w = A.pm[a];
    c[0] += w * (A.o11 * x + A.o12 * y + A.o13 * z);
    c[1] += w * (A.o22 * y + A.o23 * z);
    c[2] += w * (A.o33 * z);
  }
  A.grp[gi] = c[0];
  A.grp[A.G + gi] = c[1];
  A.grp[2 * A.G + gi] = c[2];
  A.gpos[gi] = make_double4(c[0], c[1], c[2], 0.0);
  for (int a = a0; a < a0 + n; a++) {
    const double x = A.x[a], y = A.x[N + a], z = A.x[2 * N + a];
    const double dx = (A.o11 * x + A.o12 * y + A.o13 * z) - c[0];
    const double dy = (A.o22 * y + A.o23 * z) - c[1];
    const double dz = (A.o33 * z) - c[2];
    A.aoff[a] = make_float4((float)(A.c11 * dx + A.c12 * dy + A.c13 * dz), (float)(A.c22 * dy + A.c23 * dz),
                            (float)(A.c33 * dz), A.q[a]);
  }
}

// The molecule kinds of the drift and kick kernels: the solvers of a rigid
// three-site molecule and of a star cluster index their arrays by
// constants, so those arrays stay in registers; the general solvers index
// them by constraint (local memory)
enum { MK_GENERAL = 0, MK_W3 = 1, MK_STAR = 2 };

// correc (v += f dt/2m) from the fixed-point level accumulators, then RATTLE,
// for one small molecule of kind KIND
template <int KIND>
__device__ __forceinline__ void kick_molecule(const MolArgs& A, const int4 m) {
  const int N = A.N;
  constexpr bool W3 = KIND == MK_W3;
  const int na = W3 ? 3 : m.y;
  int gat[SMA];
  double im[SMA];
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    gat[a] = a < na ? sm_atom(A, m, a) : 0;
    im[a] = a < na ? __ldg(&A.invm[gat[a]]) : 0.0;
  }
  pdl_enter();
  double x[SMA][3], v[SMA][3];
  const int nlev = (m.w & NOINTRA) ? LN1 : NLV;
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    if (a < na) {
      const int g = gat[a];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        x[a][d] = A.x[d * N + g];
        v[a][d] = A.v[d * N + g] + kick_dv(A, d * N + g, nlev) * im[a];
      }
    } else {
#pragma unroll
      for (int d = 0; d < 3; d++) x[a][d] = v[a][d] = 0.0;
    }
  }
  bool ok;
  if constexpr (W3)
    ok = rattle3(x, v, im);
  else if constexpr (KIND == MK_STAR)
    ok = rattle_star_n(m.w & 0xff, x, v, im);
  else
    ok = rattle_small(x, v, im, A.cloc + m.z, m.w & 0xff);
  if (!ok) atomicOr(A.flag, 1);
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    if (a < na) {
      const int g = gat[a];
#pragma unroll
      for (int d = 0; d < 3; d++) A.v[d * N + g] = v[a][d];
    }
  }
}

// Threads [0, nsm) take one small molecule each, the rest one free atom.
__global__ void k_kick(const MolArgs A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = A.N;
  if (t < A.nsm) {
    const int4 m = __ldg(&A.sm[t]);
    if (m.w & MOL3)
      kick_molecule<MK_W3>(A, m);
    else if (m.w & STAR)
      kick_molecule<MK_STAR>(A, m);
    else
      kick_molecule<MK_GENERAL>(A, m);
  } else if (t < A.nsm + A.nfree) {
    pdl_enter();
    const int g = A.free_atoms[t - A.nsm];
    const double im = A.invm[g];
    A.v[g] += kick_dv(A, g) * im;
    A.v[N + g] += kick_dv(A, N + g) * im;
    A.v[2 * N + g] += kick_dv(A, 2 * N + g) * im;
  } else {
    pdl_enter();
  }
}

// One small constrained molecule (thread t): verlet drift (src/verlet.f) +
// SHAKE + RATTLE, then the scaled frame, group centres (appbou) and the
// pair-kernel inputs of its groups, for a molecule of kind KIND (a rigid
// three-site molecule: SETTLE or Newton SHAKE; a star cluster; the general
// small molecule).
template <int KIND, bool TH>
__device__ __forceinline__ void drift_molecule(const MolArgs& A, int t, const int4 m) {
  constexpr bool W3 = KIND == MK_W3;
  const int N = A.N;
  const double dt = A.dt;
  const int na = W3 ? 3 : m.y;
  // The molecule's topology, masses, charges and constraint lengths are
  // written by no kernel: they are loaded together, before the wait for the
  // preceding grid, so that one memory round trip covers them.
  const int2 gg = A.groups ? __ldg(&A.smg[t]) : make_int2(0, 0);
  const int2 mg0 = gg.y > 0 ? __ldg(&A.gmeta[gg.x]) : make_int2(0, 0);
  const int nlev = (m.w & NOINTRA) ? LN1 : NLV;
  int gat[SMA];
  double im[SMA], pmv[SMA];
  float qv[SMA];
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    gat[a] = a < na ? sm_atom(A, m, a) : 0;
    im[a] = a < na ? __ldg(&A.invm[gat[a]]) : 0.0;
    pmv[a] = (a < na && gg.y > 0) ? __ldg(&A.pm[m.x + a]) : 0.0;
    qv[a] = (a < na && gg.y > 0) ? __ldg(&A.q[m.x + a]) : 0.f;
  }
  double L2v[3] = {0.0, 0.0, 0.0};
  if constexpr (W3)
#pragma unroll
    for (int k = 0; k < 3; k++) L2v[k] = __ldg(&A.dss[m.z + k]);
  pdl_enter();
  double x[SMA][3], xo[SMA][3], v[SMA][3], fh[SMA][3];
  // positions, velocities, the kick's level forces and the verlet step's
  // N0 force (as 0.5 dt f / m), all issued before any arithmetic
  const bool vf = A.fv && nlev == NLV;
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    if (a < na) {
      const int g = gat[a];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        xo[a][d] = A.x[d * N + g];
        v[a][d] = A.v[d * N + g];
        if (!TH && A.kick) v[a][d] += kick_dv(A, d * N + g, nlev) * im[a];
        fh[a][d] = vf ? fixd(A.fv[d * N + g]) : 0.0;
      }
    } else {
#pragma unroll
      for (int d = 0; d < 3; d++) x[a][d] = xo[a][d] = v[a][d] = fh[a][d] = 0.0;
    }
  }
  if constexpr (TH) {
    // the M step's start sandwich under thermostats, then the kick
    const bool big = (m.w & CLUSTER) != 0;
    const int p = big ? A.abm[gat[0]] : 0;
    const double sc = A.th->s[0], sk = A.th->s[A.tcls[gat[0]]];
    double M = 0.0;
#pragma unroll
    for (int a = 0; a < SMA; a++)
      if (a < na) M += 1.0 / im[a];
    double V[3], F[3];
    const double iM = big ? 1.0 / A.bmass[p] : 1.0 / M;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (big) {
        V[d] = A.vcur[3 * p + d];
        F[d] = fixd(A.msum[(size_t)p * TH_NS + 9 + d]);
      } else {
        double tv = 0.0, tf = 0.0;
#pragma unroll
        for (int a = 0; a < SMA; a++)
          if (a < na) {
            tv += v[a][d] / im[a];
            tf += fixd(A.fk[LM][d * N + gat[a]]);
          }
        V[d] = tv / M;
        F[d] = tf;
      }
    }
#pragma unroll
    for (int a = 0; a < SMA; a++)
      if (a < na)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          v[a][d] = sandwich(v[a][d], fixd(A.fk[LM][d * N + gat[a]]), im[a], V[d], F[d], iM, sk, sc, A.tcm);
          if (A.kick) v[a][d] += kick_dv(A, d * N + gat[a], nlev) * im[a];
        }
  }
  const int nc = m.w & 0xff;
  // RATTLE of the kicked velocities (rattle_correc after correc).  A rigid
  // three-site molecule skips it: SETTLE and the Newton SHAKE move the
  // atoms along the old bonds only, so a velocity change along those bonds
  // leaves the constrained positions, and the velocities (x_new - x_old)/dt
  // they leave, as they were (to rounding)
  if constexpr (!W3) {
    if ((A.kick || TH) && nc > 0) {
      bool ok;
      if constexpr (KIND == MK_STAR)
        ok = rattle_star_n(nc, xo, v, im);
      else
        ok = rattle_small(xo, v, im, A.cloc + m.z, nc);
      if (!ok) atomicOr(A.flag, 1);
    }
  }
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    if (a < na) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double f = fh[a][d];
        x[a][d] = xo[a][d] + dt * v[a][d] + f * 0.5 * dt * dt * im[a];
        v[a][d] += f * 0.5 * dt * im[a];
      }
    }
  }
  if constexpr (W3) {
    // isosceles with equal masses at the base: SETTLE, else Newton steps
    const bool iso = im[1] == im[2] && fabs(L2v[0] - L2v[1]) <= 1e-12 * L2v[0];
    if (!(iso ? settle3(x, xo, v, im, L2v, A.idt) : shake3(x, xo, v, im, L2v, dt, A.tol))) atomicOr(A.flag, 1);
    if (!rattle3(x, v, im)) atomicOr(A.flag, 1);
  } else if constexpr (KIND == MK_STAR) {
    if (!shake_star_n(nc, x, xo, v, im, A.dss + m.z, A.idt, A.tol)) atomicOr(A.flag, 1);
    if (!rattle_star_n(nc, x, v, im)) atomicOr(A.flag, 1);
  } else if (nc > 0) {
    if (!shake_small(x, xo, v, im, A.cloc + m.z, A.dss + m.z, nc, dt, A.tol)) atomicOr(A.flag, 1);
    if (!rattle_small(x, v, im, A.cloc + m.z, nc)) atomicOr(A.flag, 1);
  }
  double s[SMA][3];
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    if (a < na) {
      const int g = gat[a];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        A.x[d * N + g] = x[a][d];
        A.xo[d * N + g] = xo[a][d];
        A.v[d * N + g] = v[a][d];
#pragma unroll
        for (int l = 0; l < NLV; l++)
          if (l < nlev && A.fz[l]) A.fz[l][d * N + g] = 0ull;
      }
      s[a][0] = A.o11 * x[a][0] + A.o12 * x[a][1] + A.o13 * x[a][2];
      s[a][1] = A.o22 * x[a][1] + A.o23 * x[a][2];
      s[a][2] = A.o33 * x[a][2];
    }
  }
  for (int gi = gg.x; gi < gg.x + gg.y; gi++) {
    const int2 mg = gi == gg.x ? mg0 : __ldg(&A.gmeta[gi]);
    double c[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < SMA; a++) {
      const int ga = m.x + a;
      if (a < na && ga >= mg.x && ga < mg.x + (mg.y & 0xff)) {
        const double w = pmv[a];
        c[0] += w * s[a][0];
        c[1] += w * s[a][1];
        c[2] += w * s[a][2];
      }
    }
    A.grp[gi] = c[0];
    A.grp[A.G + gi] = c[1];
    A.grp[2 * A.G + gi] = c[2];
    A.gpos[gi] = make_double4(c[0], c[1], c[2], 0.0);
#pragma unroll
    for (int a = 0; a < SMA; a++) {
      const int ga = m.x + a;
      if (a < na && ga >= mg.x && ga < mg.x + (mg.y & 0xff)) {
        const double dx = s[a][0] - c[0], dy = s[a][1] - c[1], dz = s[a][2] - c[2];
        A.aoff[ga] = make_float4((float)(A.c11 * dx + A.c12 * dy + A.c13 * dz), (float)(A.c22 * dy + A.c23 * dz),
                                 (float)(A.c33 * dz), qv[a]);
      }
    }
  }
}

// verlet drift + SHAKE + RATTLE of small molecules (drift_molecule); free
// atoms drift here and get their groups in k_free_groups.
template <bool TH>
__global__ void k_drift(const MolArgs A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = A.dt;
  if (t < A.nsm) {
    const int4 m = __ldg(&A.sm[t]);
    if (m.w & MOL3)
      drift_molecule<MK_W3, TH>(A, t, m);
    else if (m.w & STAR)
      drift_molecule<MK_STAR, TH>(A, t, m);
    else
      drift_molecule<MK_GENERAL, TH>(A, t, m);
  } else if (t < A.nsm + A.ndg) {
    pdl_enter();
    // a group of an unconstrained molecule: its atoms, then its centre
    const int gi = A.drift_groups[t - A.nsm];
    const int2 mg = A.gmeta[gi];
    for (int a = mg.x; a < mg.x + (mg.y & 0xff); a++) drift_atom<TH>(A, a, dt);
    if (A.groups) group_centre(A, gi);
  } else if (t < A.nsm + A.ndg + A.nda) {
    pdl_enter();
    drift_atom<TH>(A, A.drift_atoms[t - A.nsm - A.ndg], dt);
  } else {
    pdl_enter();
  }
}

// group centres and pair-kernel inputs of the groups of large constrained
// molecules, after their iterative SHAKE
__global__ void k_free_groups(const MolArgs A) {
  pdl_enter();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.nfreeg) return;
  group_centre(A, A.free_groups[t]);
}

struct ConsArgs {
  int nmol;           // large constrained molecules
  const int* cstart;  // [nmol+1]
  const int2* cab;    // constraint atoms (global)
  const double* dss;
  const double* invm;
  int N;
  double* x;
  const double* xo;
  double* v;
  double dt;
  double tol;
  int maxit;
  int* flag;
};

// iterative SHAKE (src/rattle_verlet.f SHAKE branch) for large molecules
__global__ void k_shake_big(const ConsArgs A) {
  pdl_enter();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= A.nmol) return;
  const int c0 = A.cstart[m], c1 = A.cstart[m + 1];
  const double dti = A.dt != 0.0 ? 1.0 / A.dt : 0.0;
  const int N = A.N;
  for (int it = 0; it < A.maxit; it++) {
    bool moved = false;
    for (int k = c0; k < c1; k++) {
      const int a = A.cab[k].x, b = A.cab[k].y;
      const double dx = A.x[a] - A.x[b], dy = A.x[N + a] - A.x[N + b], dz = A.x[2 * N + a] - A.x[2 * N + b];
      const double dcnt = dx * dx + dy * dy + dz * dz - A.dss[k];
      if (fabs(dcnt) >= A.tol) {
        moved = true;
        const double rx = A.xo[a] - A.xo[b], ry = A.xo[N + a] - A.xo[N + b], rz = A.xo[2 * N + a] - A.xo[2 * N + b];
        const double ia = A.invm[a], ib = A.invm[b];
        const double gg = dcnt / ((dx * rx + dy * ry + dz * rz) * 2.0 * (ia + ib));
        const double ga = -gg * ia, gb = gg * ib;
        A.x[a] += rx * ga;
        A.x[b] += rx * gb;
        A.x[N + a] += ry * ga;
        A.x[N + b] += ry * gb;
        A.x[2 * N + a] += rz * ga;
        A.x[2 * N + b] += rz * gb;
        A.v[a] += rx * ga * dti;
        A.v[b] += rx * gb * dti;
        A.v[N + a] += ry * ga * dti;
        A.v[N + b] += ry * gb * dti;
        A.v[2 * N + a] += rz * ga * dti;
        A.v[2 * N + b] += rz * gb * dti;
      }
    }
    if (!moved) return;
  }
  atomicOr(A.flag, 1);
}

// iterative RATTLE velocity step (src/rattle_correc.f) for large molecules
__global__ void k_rattle_big(const ConsArgs A) {
  pdl_enter();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= A.nmol) return;
  const int c0 = A.cstart[m], c1 = A.cstart[m + 1];
  const int N = A.N;
  for (int it = 0; it < A.maxit; it++) {
    bool moved = false;
    for (int k = c0; k < c1; k++) {
      const int a = A.cab[k].x, b = A.cab[k].y;
      const double rx = A.x[a] - A.x[b], ry = A.x[N + a] - A.x[N + b], rz = A.x[2 * N + a] - A.x[2 * N + b];
      const double vx = A.v[a] - A.v[b], vy = A.v[N + a] - A.v[N + b], vz = A.v[2 * N + a] - A.v[2 * N + b];
      const double dpp = rx * vx + ry * vy + rz * vz;
      if (fabs(dpp) > A.tol) {
        moved = true;
        const double ia = A.invm[a], ib = A.invm[b];
        const double g = -dpp / (A.dss[k] * (ia + ib));
        A.v[a] += g * ia * rx;
        A.v[b] -= g * ib * rx;
        A.v[N + a] += g * ia * ry;
        A.v[N + b] -= g * ib * ry;
        A.v[2 * N + a] += g * ia * rz;
        A.v[2 * N + b] -= g * ib * rz;
      }
    }
    if (!moved) return;
  }
  atomicOr(A.flag, 1);
}


// The energy record of an energy step (ORAC_MD_REC doubles, the layout
// orac_gpu_md_run returns) into the context's ring: [0] record number,
// [1] kinetic, [2..7] M, L, H LJ and Coulomb, [8] SPME, [9] the constant
// (self energy), [10] total, [11] status flags, [12] bonded, [13] 1-4 and
// intra-group pairs, [14] erf corrections, [15] dU/dlambda (alchemy), the
// REM segment's nonbonded energy (REM), the work of a non-equilibrium run, or
// for a standard context the thermostats' energy (Nose-Hoover thermostats
// add it to [10] in every case).
__global__ void k_record(const double* __restrict__ e, const int* __restrict__ flag, double econst, double self_dudl,
                         int var, double* __restrict__ ring, int cap, unsigned long long* __restrict__ n,
                         const NeDev* __restrict__ ne, const ThermoDev* __restrict__ th) {
  pdl_enter();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const unsigned long long k = *n;
  double* r = ring + (size_t)ORAC_MD_REC * (size_t)(k % (unsigned long long)cap);
  r[0] = (double)(k + 1);
  r[1] = e[40];
  r[2] = e[4] + e[0] + e[6];
  r[3] = e[5] + e[1] + e[7];
  r[4] = e[12] + e[8] + e[14];
  r[5] = e[13] + e[9] + e[15];
  r[6] = e[20] + e[16] + e[22];
  r[7] = e[21] + e[17] + e[23];
  r[8] = 0.5 * e[24];
  r[9] = econst;
  double b = 0.0, p = 0.0, c = 0.0, d = 0.0;
  for (int q = 41; q < 49; q++) b += e[q];  // bonded (E_BOND..E_14)
  for (int q = 49; q < 57; q++) p += e[q];  // 1-4 and intra-group (E_14..E_ERF)
  for (int q = 57; q < 73; q++) c += e[q];  // erf corrections (E_ERF..E_DUDL)
  c += e[80] + e[81];                       // ferrf_alchemy_add (E_AQQ)
  if (var == 2) {  // alchemy: dU/dlambda of every term
    for (int q = 73; q < 80; q++) d += e[q];
    d += self_dudl;
  } else if (var == 1) {  // REM: the segment energy of the three shells (rem_pot(3))
    for (int q = 73; q < 76; q++) d += e[q];
  } else if (var == 3) {  // a non-equilibrium schedule: the work so far (wrk_alchemy)
    d = ne->wrk;
  }
  r[12] = b;
  r[13] = p;
  r[14] = c;
  r[15] = d;
  r[10] = r[1] + r[2] + r[3] + r[4] + r[5] + r[6] + r[7] + r[8] + r[9] + r[12] + r[13] + r[14];
  if (th) {  // the thermostats' energy (comp_thermos_energy): the extended system's total
    double et = 0.0;
    for (int k = 0; k < 3; k++) et += th->ndfkt[k] * th->eta[k] + 0.5 * th->q[k] * th->etap[k] * th->etap[k];
    r[10] += et;
    if (var == 0) r[15] = et;  // where the column has no other use
  }
  r[11] = (double)*flag;
  *n = k + 1;
}

__global__ void k_ekin(int N, const double* __restrict__ v, const double* __restrict__ invm, double* __restrict__ out) {
  pdl_enter();
  __shared__ double s[8];
  double e = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x)
    e += 0.5 / invm[t] * (v[t] * v[t] + v[N + t] * v[N + t] + v[2 * N + t] * v[2 * N + t]);
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) x += s[k];
    atomicAdd(out, x);
  }
}

// ---------------------------------------------------------------------------
// ORAC's Nose-Hoover thermostats (THERMOS) at the M level
// (src/mtsmd.f:2556-2618, 2932, 3109-3170).  ORAC keeps each molecule's
// centre-of-mass velocity V apart from its atoms' velocities u relative to
// it (comp_fcm, src/comp_fcm.f); the driver keeps atomic velocities v = V + u
// and splits them where a thermostat acts.  The M half kick at either end
// of an M step sits between two scalings (correc_exp_scale): V by
// s_c = exp(-tm/4 etap1), u by s_k = exp(-tm/4 etap_k) (k 2: solute, 3:
// solvent), so with c = tm/2 and F the molecule's M force
//   v <- s_k (s_k (v - V) + c (f/m - F/M)) + s_c (s_c V + c F/M),
// then RATTLE (its impulses move no centre of mass and it commutes with the
// split scaling, so one projection after the sandwich is the same).  The
// thermostats' velocities follow comp_thermos_forces + correc_etap twice at
// each end of the M step: etap_k += tm/4 (tto_k - ndf_k kT) / Q_k with
// tto = sum M V^2 over molecules, sum m u^2 over solute and over solvent
// atoms, taken after the end sandwich (K1) and before the start sandwich
// (K2, after the L and H kicks that come between them).

// one warp per block of k_thermo (its threads' chains are long: the blocks
// spread over the SMs); k_mol_sums takes 64 atoms of one molecule per block
constexpr int TH_BLOCK = 32;
constexpr int TS_BLOCK = 64;
constexpr int TH_CHUNK = 64;

struct ThermoArgs {
  int N, nsm, nfree, nbm;
  const int4* sm;
  const int2* cloc;
  const int* sm_atoms;
  const int* free_atoms;
  const double* x;
  double* v;
  const double* invm;
  const int* cls;       // [N] 1 solute, 2 solvent: the thermostat of the atom's relative velocity
  const int* abm;       // [N] molecule of the atom among those outside small molecules, or -1
  const int4* bchunk;   // k_mol_sums blocks: molecule, first atom, atoms (at most TH_CHUNK)
  const double* bmass;  // [nbm]
  unsigned long long* msum;  // [nbm][TH_NS] fixed point
  double* vcur;         // [nbm][3] centre-of-mass velocity the pass leaves (the drift's start sandwich reads it)
  const unsigned long long* f[NLV];
  // the end half kicks of N0 (c0) and N1 (c1), the end sandwich with the M
  // half kick cm, K1; then kicks of L (cl) and H (ch) and K2 (the start
  // sandwich follows in the drift, k_drift<true>)
  double c0, c1, cm, cl, ch;
  int end, k2;
  int lvmask;  // levels k_mol_sums sums (bit q: N0, N1, M, L, H)
  ThermoDev* th;
  double* part;  // [blocks][6]: K1 and K2 of each block
  int* flag;
};

__device__ __forceinline__ double fixf(const unsigned long long* f, int i) { return f ? fixd(f[i]) : 0.0; }

// the q-th level of the sums: N0, N1, M, L, H
__device__ __forceinline__ int th_level(int q) { return LN0 - q; }

// sum j of molecule p
__device__ __forceinline__ double msv(const ThermoArgs& A, int p, int j) { return fixd(A.msum[(size_t)p * TH_NS + j]); }

// one block per chunk of at most TH_CHUNK atoms of one molecule: the
// chunk's integer sums, added into the molecule's by one atomic each
__global__ void __launch_bounds__(TS_BLOCK) k_mol_sums(const ThermoArgs A) {
  const int4 c = __ldg(&A.bchunk[blockIdx.x]);
  pdl_enter();
  const int N = A.N;
  unsigned long long s[TH_NS];
#pragma unroll
  for (int j = 0; j < TH_NS; j++) s[j] = 0ull;
  for (int a = c.y + threadIdx.x; a < c.y + c.z; a += blockDim.x) {
    const double m = 1.0 / A.invm[a];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      s[d] += (unsigned long long)__double2ll_rn(m * A.v[d * N + a] * ORAC_FSCALE);
#pragma unroll
      for (int q = 0; q < 5; q++)
        if ((A.lvmask >> q) & 1) s[3 + 3 * q + d] += A.f[th_level(q)][d * N + a];
    }
  }
  __shared__ unsigned long long sh[TS_BLOCK / 32][TH_NS];
#pragma unroll
  for (int j = 0; j < TH_NS; j++) {
    unsigned long long x = s[j];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5][j] = x;
  }
  __syncthreads();
  const int j = threadIdx.x;
  if (j < TH_NS && (j < 3 || ((A.lvmask >> ((j - 3) / 3)) & 1))) {
    unsigned long long x = 0ull;
    for (int w = 0; w < TS_BLOCK / 32; w++) x += sh[w][j];
    atomicAdd(&A.msum[(size_t)c.x * TH_NS + j], x);
  }
}

// centre-of-mass velocity of molecule p (outside the small molecules) at the
// stages of the pass, from its sums: Va after the end kicks, V1 after
// the end sandwich, V2 after the L and H kicks; FM its M force
struct BigStages {
  double Va[3], V1[3], V2[3], FM[3], iM;
};

__device__ __forceinline__ void big_stages(const ThermoArgs& A, int p, const double* sc, BigStages& B) {
  B.iM = 1.0 / A.bmass[p];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    B.Va[d] = msv(A, p, d) * B.iM + (A.c0 * msv(A, p, 3 + d) + A.c1 * msv(A, p, 6 + d)) * B.iM;
    B.FM[d] = msv(A, p, 9 + d);
    B.V1[d] = A.end ? sc[0] * (sc[0] * B.Va[d] + A.cm * B.FM[d] * B.iM) : B.Va[d];
    B.V2[d] = B.V1[d] + (A.cl * msv(A, p, 12 + d) + A.ch * msv(A, p, 15 + d)) * B.iM;
  }
}

// atom a of entry m (a cluster lists its atoms in sm_atoms)
__device__ __forceinline__ int th_atom(const ThermoArgs& A, const int4& m, int a) {
  return (m.w & CLUSTER) ? A.sm_atoms[m.x + a] : m.x + a;
}

template <int KIND>
__device__ __forceinline__ bool th_rattle(const ThermoArgs& A, const int4& m, const double x[SMA][3], double v[SMA][3],
                                          const double im[SMA]) {
  const int nc = m.w & 0xff;
  if constexpr (KIND == MK_W3)
    return rattle3(x, v, im);
  else if constexpr (KIND == MK_STAR)
    return rattle_star_n(nc, x, v, im);
  else
    return rattle_small(const_cast<double(*)[3]>(x), v, im, A.cloc + m.z, nc);
}

// one small molecule or constraint cluster (entry m) of kind KIND: its share
// of the pass and of K1 and K2
template <int KIND>
__device__ __forceinline__ void thermo_entry(const ThermoArgs& A, const int4 m, double k1[3], double k2[3]) {
  const int N = A.N;
  constexpr bool W3 = KIND == MK_W3;
  const int na = W3 ? 3 : m.y;
  const bool big = (m.w & CLUSTER) != 0;
  int gat[SMA];
  double im[SMA];
#pragma unroll
  for (int a = 0; a < SMA; a++) {
    gat[a] = a < na ? th_atom(A, m, a) : 0;
    im[a] = a < na ? __ldg(&A.invm[gat[a]]) : 0.0;
  }
  const int c = __ldg(&A.cls[gat[0]]);
  const int p = big ? __ldg(&A.abm[gat[0]]) : -1;
  pdl_enter();
  double x[SMA][3], v[SMA][3];
  double M = 0.0;
#pragma unroll
  for (int a = 0; a < SMA; a++) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      x[a][d] = a < na ? A.x[d * N + gat[a]] : 0.0;
      v[a][d] = a < na ? A.v[d * N + gat[a]] : 0.0;
    }
    if (a < na) M += 1.0 / im[a];
  }
  const double sc = A.th->s[0], sk = A.th->s[c];
  // centre-of-mass velocity and M force of a small molecule from its atoms
  auto com = [&](double V[3]) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double t = 0.0;
#pragma unroll
      for (int a = 0; a < SMA; a++)
        if (a < na) t += v[a][d] / im[a];
      V[d] = t / M;
    }
  };
  auto fsum = [&](double F[3]) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double t = 0.0;
#pragma unroll
      for (int a = 0; a < SMA; a++)
        if (a < na) t += fixf(A.f[LM], d * N + gat[a]);
      F[d] = t;
    }
  };
  // relative kinetic term sum m |v - V|^2 and, for a small molecule, M |V|^2
  auto kin = [&](const double V[3], double k[3]) {
    double u2 = 0.0;
#pragma unroll
    for (int a = 0; a < SMA; a++)
      if (a < na) {
        double t = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) t += (v[a][d] - V[d]) * (v[a][d] - V[d]);
        u2 += t / im[a];
      }
    k[c] += u2;
    if (!big) k[0] += M * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
  };
  bool ok = true;
  {
    BigStages B;
    if (big) big_stages(A, p, A.th->s, B);
    if (A.end) {
#pragma unroll
      for (int a = 0; a < SMA; a++)
        if (a < na)
#pragma unroll
          for (int d = 0; d < 3; d++)
            v[a][d] += (A.c0 * fixf(A.f[LN0], d * N + gat[a]) + A.c1 * fixf(A.f[LN1], d * N + gat[a])) * im[a];
      double Va[3], F[3];
      if (big) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
          Va[d] = B.Va[d];
          F[d] = B.FM[d];
        }
      } else {
        com(Va);
        fsum(F);
      }
      const double iM = big ? B.iM : 1.0 / M;
#pragma unroll
      for (int a = 0; a < SMA; a++)
        if (a < na)
#pragma unroll
          for (int d = 0; d < 3; d++)
            v[a][d] = sandwich(v[a][d], fixf(A.f[LM], d * N + gat[a]), im[a], Va[d], F[d], iM, sk, sc, A.cm);
      ok = th_rattle<KIND>(A, m, x, v, im);
      double V1[3];
      if (big) {
#pragma unroll
        for (int d = 0; d < 3; d++) V1[d] = B.V1[d];
      } else {
        com(V1);
      }
      kin(V1, k1);
    }
    if (A.cl != 0.0 || A.ch != 0.0) {
#pragma unroll
      for (int a = 0; a < SMA; a++)
        if (a < na)
#pragma unroll
          for (int d = 0; d < 3; d++)
            v[a][d] += (A.cl * fixf(A.f[LL], d * N + gat[a]) + A.ch * fixf(A.f[LH], d * N + gat[a])) * im[a];
      ok = th_rattle<KIND>(A, m, x, v, im) && ok;
    }
    if (A.k2) {
      double V2[3];
      if (big) {
#pragma unroll
        for (int d = 0; d < 3; d++) V2[d] = B.V2[d];
      } else {
        com(V2);
      }
      kin(V2, k2);
    }
  }
  if (!ok) atomicOr(A.flag, 1);
#pragma unroll
  for (int a = 0; a < SMA; a++)
    if (a < na)
#pragma unroll
      for (int d = 0; d < 3; d++) A.v[d * N + gat[a]] = v[a][d];
}

// correc_etap (src/correc_etap.f) with tto from comp_thermos_forces
__device__ __forceinline__ void th_etap(ThermoDev& T, const double K[3]) {
  for (int k = 0; k < 3; k++) {
    if (fabs(T.q[k]) > 1.0e-7)
      T.etap[k] += T.tm4 * (K[k] - T.ndfkt[k]) / T.q[k];
    else
      T.etap[k] = 0.0;
  }
}

// Threads [0, nsm) take one small molecule or constraint cluster each,
// [nsm, nsm + nfree) one atom outside them, the next nbm one molecule
// outside the small ones (its centre-of-mass terms).  Each block leaves its
// K1 and K2 sums in part; the last block to finish adds
// them in block order (the same result at every run) and moves the
// thermostats: eta += tm etap (verlet_free_eta, once per M step), etap
// twice from K1 (the end of the M step), twice from K2 (the start of the
// next), and the scales of the next sandwiches.
__global__ void __launch_bounds__(TH_BLOCK) k_thermo(const ThermoArgs A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = A.N;
  double k1[3] = {0.0, 0.0, 0.0}, k2[3] = {0.0, 0.0, 0.0};
  if (t < A.nsm) {
    const int4 m = __ldg(&A.sm[t]);
    if (m.w & MOL3)
      thermo_entry<MK_W3>(A, m, k1, k2);
    else if (m.w & STAR)
      thermo_entry<MK_STAR>(A, m, k1, k2);
    else
      thermo_entry<MK_GENERAL>(A, m, k1, k2);
  } else if (t < A.nsm + A.nfree) {
    const int g = __ldg(&A.free_atoms[t - A.nsm]);
    const double im = __ldg(&A.invm[g]);
    const int c = __ldg(&A.cls[g]);
    const int p = __ldg(&A.abm[g]);
    pdl_enter();
    const double sc = A.th->s[0], sk = A.th->s[c];
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; d++) v[d] = A.v[d * N + g];
    {
      BigStages B;
      big_stages(A, p, A.th->s, B);
      if (A.end) {
        double u2 = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          v[d] += (A.c0 * fixf(A.f[LN0], d * N + g) + A.c1 * fixf(A.f[LN1], d * N + g)) * im;
          v[d] = sandwich(v[d], fixf(A.f[LM], d * N + g), im, B.Va[d], B.FM[d], B.iM, sk, sc, A.cm);
          u2 += (v[d] - B.V1[d]) * (v[d] - B.V1[d]);
        }
        k1[c] += u2 / im;
      }
      double u2 = 0.0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        v[d] += (A.cl * fixf(A.f[LL], d * N + g) + A.ch * fixf(A.f[LH], d * N + g)) * im;
        u2 += (v[d] - B.V2[d]) * (v[d] - B.V2[d]);
      }
      if (A.k2) k2[c] += u2 / im;
    }
#pragma unroll
    for (int d = 0; d < 3; d++) A.v[d * N + g] = v[d];
  } else if (t < A.nsm + A.nfree + A.nbm) {
    pdl_enter();
    {
      const int p = t - A.nsm - A.nfree;
      BigStages B;
      big_stages(A, p, A.th->s, B);
      const double M = A.bmass[p];
      if (A.end) k1[0] += M * (B.V1[0] * B.V1[0] + B.V1[1] * B.V1[1] + B.V1[2] * B.V1[2]);
      if (A.k2) k2[0] += M * (B.V2[0] * B.V2[0] + B.V2[1] * B.V2[1] + B.V2[2] * B.V2[2]);
#pragma unroll
      for (int d = 0; d < 3; d++) A.vcur[3 * p + d] = B.V2[d];
    }
  } else {
    pdl_enter();
  }
  __shared__ double red[6][TH_BLOCK / 32];
  __shared__ bool last;
  double kk[6] = {k1[0], k1[1], k1[2], k2[0], k2[1], k2[2]};
#pragma unroll
  for (int j = 0; j < 6; j++) {
    double x = kk[j];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 0; j < 6; j++) {
      double x = 0.0;
      for (int w = 0; w < TH_BLOCK / 32; w++) x += red[j][w];
      A.part[6 * blockIdx.x + j] = x;
    }
    __threadfence();
    last = atomicAdd(&A.th->count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the blocks' sums: lane l adds blocks l, l + 32, ... in order, then a
  // fixed butterfly over the lanes (the same result at every run)
  const volatile double* P = A.part;
  double K[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (threadIdx.x < 32)
    for (unsigned b = threadIdx.x; b < gridDim.x; b += 32)
#pragma unroll
      for (int j = 0; j < 6; j++) K[j] += P[6 * b + j];
#pragma unroll
  for (int j = 0; j < 6; j++)
    for (int o = 16; o > 0; o >>= 1) K[j] += __shfl_xor_sync(0xffffffffu, K[j], o);
  if (threadIdx.x != 0) return;
  const double K1[3] = {K[0], K[1], K[2]}, K2[3] = {K[3], K[4], K[5]};
  ThermoDev& T = *A.th;
  if (A.end) {
    for (int k = 0; k < 3; k++) T.eta[k] += T.tm * T.etap[k];
    th_etap(T, K1);
    th_etap(T, K1);
  }
  if (A.k2) {
    th_etap(T, K2);
    th_etap(T, K2);
  }
  for (int k = 0; k < 3; k++) T.s[k] = exp(-T.tm4 * T.etap[k]);
  T.count = 0;
}

}  // namespace

// --------------------------------------------------------------------------

struct MdState {
  bool ready = false;
  int N = 0;
  double* x = nullptr;  // [3N] Cartesian
  double* v = nullptr;
  double* xo = nullptr;
  // level accumulators H, L, M, N1, N0 (N1/N0 only with intramolecular terms)
  unsigned long long* ffix[NLV] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  bool has_n0 = false, has_n1 = false;
  double* invm = nullptr;
  double* pm = nullptr;
  // small constrained molecules
  int nsm = 0;
  int4* sm = nullptr;
  int2* smg = nullptr;
  int2* cloc = nullptr;
  double* cdss = nullptr;
  // free atoms and groups: all atoms outside small molecules (k_kick), the
  // drift's groups of unconstrained molecules and atoms of large constrained
  // ones, and the groups of the latter (k_free_groups)
  int nfree = 0, nfreeg = 0, ndg = 0, nda = 0;
  int* free_atoms = nullptr;
  int* free_groups = nullptr;
  int* drift_groups = nullptr;
  int* drift_atoms = nullptr;
  int* sm_atoms = nullptr;
  // large constrained molecules
  int nbig = 0;
  int* bstart = nullptr;
  int2* bcab = nullptr;
  double* bdss = nullptr;
  // energies: [0..7] M, [8..15] L, [16..23] H (ORAC order), [24..39] SPME
  // eout, [40] ekin, [E_BOND..+8) bonded, [E_14..+4) 1-4, [E_GRP..+4)
  // intra-group, [E_ERF..+16) erf corrections (bonds, constraints, 1-3, 1-4)
  double* e = nullptr;
  int* flag = nullptr;
  // schedule
  double dth = 0;
  int lrespa = 1, mrespa = 1, n1respa = 1, n0respa = 1, nupdte = 1;
  char rshk = 'l';
  long long step = 0;
  double econst = 0;
  // captured step graphs by kind: bit 0 list update, bit 1 energy record
  cudaGraph_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraphExec_t gexec[4] = {nullptr, nullptr, nullptr, nullptr};
  unsigned graphs_gen = 0;  // ctx->param_gen when the graphs were captured
  bool graphs_shared = false;  // ctx->shared_device when the graphs were captured
  bool use_graph = true;
  int pslot[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};  // profiling event slots of each graph
  int64_t kpg[4] = {0, 0, 0, 0};                       // kernels per captured graph
  // energy records of the energy steps (MD_REC doubles each, k_record): a
  // ring of rec_cap records on the device and the count written so far
  double* rec = nullptr;
  unsigned long long* rec_n = nullptr;
  int rec_cap = 0;
  int last_kind = -1;                  // graph of the last queued step
  // second stream of the step: work that depends only on the drifted
  // positions and adds into its own level accumulators (intramolecular
  // levels, SPME with its erf corrections) runs there beside the shell pair
  // kernels; fork and join by events (captured as graph edges)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // a third stream for the L and H shells of the step's last drift
  cudaStream_t side2 = nullptr;
  cudaEvent_t ev_fork2 = nullptr, ev_join2 = nullptr;
  // status flags read back through pinned memory; flag_step is the step
  // count at the last read-back that followed a synchronisation
  int* h_flag = nullptr;
  long long flag_step = -1;
  // Nose-Hoover thermostats (k_thermo): device state, per-block partial
  // sums, the molecules outside the small ones (ranges, masses, sums,
  // centre-of-mass velocities), the atoms' thermostat and molecule
  ThermoDev* th = nullptr;
  int th_blocks = 0, nbm = 0;
  double* tpart = nullptr;
  int4* bchunk = nullptr;
  int nchunk = 0;
  double* bmass = nullptr;
  unsigned long long* msum = nullptr;
  double* vcur = nullptr;
  int* tcls = nullptr;
  int* abm = nullptr;
  int th_ndf[3] = {0, 0, 0};
  double th_tm = 0.0;  // the M step
};

static MdState* md_of(orac_gpu_ctx* ctx) {
  if (!ctx->md) ctx->md = new MdState();
  return ctx->md;
}

void md_destroy(orac_gpu_ctx* ctx) {
  MdState* S = ctx->md;
  if (!S) return;
  for (int k = 0; k < 4; k++) {
    if (S->gexec[k]) cudaGraphExecDestroy(S->gexec[k]);
    if (S->graph[k]) cudaGraphDestroy(S->graph[k]);
  }
  if (S->h_flag) cudaFreeHost(S->h_flag);
  if (S->ev_fork) cudaEventDestroy(S->ev_fork);
  if (S->ev_join) cudaEventDestroy(S->ev_join);
  if (S->side) cudaStreamDestroy(S->side);
  if (S->ev_fork2) cudaEventDestroy(S->ev_fork2);
  if (S->ev_join2) cudaEventDestroy(S->ev_join2);
  if (S->side2) cudaStreamDestroy(S->side2);
  void* ptrs[] = {S->x,         S->xo,          S->ffix[0],   S->ffix[1], S->ffix[2], S->ffix[3],
                  S->ffix[4],
                  S->invm,      S->pm,       S->sm,          S->smg,       S->cloc,    S->cdss,    S->free_atoms,
                  S->free_groups, S->bstart, S->bcab,        S->bdss,      S->e,       S->flag,
                  S->drift_groups, S->drift_atoms, S->sm_atoms, S->rec, S->rec_n, S->th, S->tpart,
                  S->bchunk, S->bmass, S->msum, S->vcur, S->tcls, S->abm};
  for (void* p : ptrs)
    if (p) dev_free(ctx, p);
  delete S;
  ctx->md = nullptr;
}

static MolArgs mol_args(orac_gpu_ctx* ctx, MdState& S, double dt) {
  MolArgs A;
  memset(&A, 0, sizeof(A));
  A.N = ctx->N;
  A.nsm = S.nsm;
  A.sm = S.sm;
  A.smg = S.smg;
  A.cloc = S.cloc;
  A.dss = S.cdss;
  A.nfree = S.nfree;
  A.free_atoms = S.free_atoms;
  A.nfreeg = S.nfreeg;
  A.free_groups = S.free_groups;
  A.ndg = S.ndg;
  A.drift_groups = S.drift_groups;
  A.nda = S.nda;
  A.drift_atoms = S.drift_atoms;
  A.sm_atoms = S.sm_atoms;
  A.x = S.x;
  A.xo = S.xo;
  A.v = S.v;
  A.invm = S.invm;
  A.pm = S.pm;
  A.q = ctx->d_aq;
  A.gmeta = ctx->d_gmeta;
  const double* o = ctx->oc;
  const double* c = ctx->co;
  A.o11 = o[0];
  A.o12 = o[3];
  A.o13 = o[6];
  A.o22 = o[4];
  A.o23 = o[7];
  A.o33 = o[8];
  A.c11 = c[0];
  A.c12 = c[3];
  A.c13 = c[6];
  A.c22 = c[4];
  A.c23 = c[7];
  A.c33 = c[8];
  A.G = ctx->G;
  A.grp = ctx->d_grp;
  A.gpos = ctx->d_gpos;
  A.aoff = ctx->d_aoff;
  A.dt = dt;
  A.idt = dt != 0.0 ? 1.0 / dt : 0.0;
  A.groups = 1;
  A.tol = 1e-12;
  A.flag = S.flag;
  return A;
}

static ConsArgs big_args(orac_gpu_ctx* ctx, MdState& S, double dt, double tol) {
  ConsArgs A;
  A.nmol = S.nbig;
  A.cstart = S.bstart;
  A.cab = S.bcab;
  A.dss = S.bdss;
  A.invm = S.invm;
  A.N = ctx->N;
  A.x = S.x;
  A.xo = S.xo;
  A.v = S.v;
  A.dt = dt;
  A.tol = tol;
  A.maxit = 5000;
  A.flag = S.flag;
  return A;
}

// dU/dlambda slots: E_DUDL + 0..2 shells, +3 SPME, +4 erf corrections,
// +5 fnb14_alchemy, +6 ferrf_alchemy_add; E_AQQ: ferrf_alchemy_add's
// energies (solute, solvent)
enum { E_BOND = 41, E_14 = 49, E_GRP = 53, E_ERF = 57, E_DUDL = 73, E_AQQ = 80, E_N = 82 };
// scratch of non-equilibrium runs: the SPME sums of chrge0, the erf
// corrections of chrgec and of chrge0, a shell's energies off energy steps
enum { E_NE0 = 82, E_NEQ = 98, E_NEQ0 = 114, E_NESH = 130, E_ALL = 160 };

// energy records kept on the device per context (the newest MD_REC_CAP)
constexpr int MD_REC_CAP = 2048;

// kick of the level accumulators with velocity factors c[l] (0: skip) + RATTLE
static void kick_fill(MolArgs& A, MdState& S, const double* c) {
  A.kick = 0;
  for (int l = 0; l < NLV; l++) {
    A.fk[l] = S.ffix[l];
    A.ck[l] = (c && S.ffix[l]) ? c[l] : 0.0;
    if (A.ck[l] != 0.0) A.kick = 1;
  }
}

static int md_kick(orac_gpu_ctx* ctx, MdState& S, const double* c) {
  MolArgs A = mol_args(ctx, S, 0.0);
  kick_fill(A, S, c);
  if (!A.kick) return ORAC_OK;
  const int n = S.nsm + S.nfree;
  int slot = -1;
  if (int rc = prof_begin(ctx, &slot, PROF_DRIFT)) return rc;
  orac_launch(k_kick, (n + 31) / 32, 32, 0, ctx->stream, A);
  CKL();
  if (int rc = prof_end(ctx, slot)) return rc;
  if (S.nbig) {
    orac_launch(k_rattle_big, (S.nbig + 127) / 128, 128, 0, ctx->stream, big_args(ctx, S, 0.0, 1e-12));
    CKL();
  }
  return ORAC_OK;
}

// [kick c + RATTLE] + verlet drift of dt (with the N0 half kick when
// present) + SHAKE + RATTLE, scaled frame and pair-kernel inputs; zeroes the
// accumulators of the levels in `zmask` (bit l) after reading them
// groups: the drift precedes a shell evaluation, so the groups of large
// molecules need their centres (the pair kernels' inputs; the
// intramolecular levels read atom positions only), as ORAC calls appbou
// only before the M forces (src/mtsmd.f:2952)
// tstart: the drift opens an M step under thermostats and applies its start
// sandwich (k_drift<true>) before the kick
static int md_drift(orac_gpu_ctx* ctx, MdState& S, double dt, const double* c, int zmask, bool groups = true,
                    bool tstart = false) {
  if (S.nbig && c) {
    // the RATTLE of large molecules is a separate kernel: kick first
    if (int rc = md_kick(ctx, S, c)) return rc;
    c = nullptr;
  }
  MolArgs A = mol_args(ctx, S, dt);
  A.groups = groups ? 1 : 0;
  kick_fill(A, S, c);
  A.fv = S.has_n0 ? S.ffix[LN0] : nullptr;
  for (int l = 0; l < NLV; l++) A.fz[l] = ((zmask >> l) & 1) ? S.ffix[l] : nullptr;
  if (tstart) {
    A.fk[LM] = S.ffix[LM];
    A.th = S.th;
    A.tcls = S.tcls;
    A.abm = S.abm;
    A.vcur = S.vcur;
    A.msum = S.msum;
    A.bmass = S.bmass;
    A.tcm = 0.5 * S.th_tm;
  }
  const int n = S.nsm + S.ndg + S.nda;
  int slot = -1;
  if (int rc = prof_begin(ctx, &slot, PROF_DRIFT)) return rc;
  if (tstart)
    orac_launch(k_drift<true>, (n + 31) / 32, 32, 0, ctx->stream, A);
  else
    orac_launch(k_drift<false>, (n + 31) / 32, 32, 0, ctx->stream, A);
  CKL();
  if (int rc = prof_end(ctx, slot)) return rc;
  if (S.nbig) {
    orac_launch(k_shake_big, (S.nbig + 127) / 128, 128, 0, ctx->stream, big_args(ctx, S, dt, 1e-8));
    CKL();
    orac_launch(k_rattle_big, (S.nbig + 127) / 128, 128, 0, ctx->stream, big_args(ctx, S, dt, 1e-12));
    CKL();
  }
  if (S.nfreeg && groups) {
    orac_launch(k_free_groups, (S.nfreeg + 31) / 32, 32, 0, ctx->stream, A);
    CKL();
  }
  return ORAC_OK;
}

// a thermostat pass (k_thermo; ThermoArgs has the coefficients) after the
// sums of the molecules outside the small ones (k_mol_sums)
static int md_thermo(orac_gpu_ctx* ctx, MdState& S, bool end, bool k2, double c0, double c1, double cm, double cl,
                     double ch) {
  ThermoArgs A;
  memset(&A, 0, sizeof(A));
  A.N = ctx->N;
  A.nsm = S.nsm;
  A.nfree = S.nfree;
  A.nbm = S.nbm;
  A.sm = S.sm;
  A.cloc = S.cloc;
  A.sm_atoms = S.sm_atoms;
  A.free_atoms = S.free_atoms;
  A.x = S.x;
  A.v = S.v;
  A.invm = S.invm;
  A.cls = S.tcls;
  A.abm = S.abm;
  A.bchunk = S.bchunk;
  A.bmass = S.bmass;
  A.msum = S.msum;
  A.vcur = S.vcur;
  for (int l = 0; l < NLV; l++) A.f[l] = S.ffix[l];
  A.c0 = c0;
  A.c1 = c1;
  A.cm = cm;
  A.cl = cl;
  A.ch = ch;
  A.end = end;
  A.k2 = k2;
  A.th = S.th;
  A.part = S.tpart;
  A.flag = S.flag;
  int slot = -1;
  if (int rc = prof_begin(ctx, &slot, PROF_DRIFT)) return rc;
  A.lvmask = (c0 != 0.0 && S.ffix[LN0] ? 1 : 0) | (c1 != 0.0 && S.ffix[LN1] ? 2 : 0) | 4 | (cl != 0.0 ? 8 : 0) |
             (ch != 0.0 ? 16 : 0);
  if (S.nbm) {
    CK(cudaMemsetAsync(S.msum, 0, sizeof(unsigned long long) * TH_NS * (size_t)S.nbm, ctx->stream));
    orac_launch(k_mol_sums, S.nchunk, TS_BLOCK, 0, ctx->stream, A);
    CKL();
  }
  orac_launch(k_thermo, S.th_blocks, TH_BLOCK, 0, ctx->stream, A);
  CKL();
  return prof_end(ctx, slot);
}

// erf corrections of the excluded pairs at the reciprocal level
// (mts_furier, src/mts_furier.f:85-141): bonds and 1-3 pairs with forces,
// 1-4 pairs with fudgec = 1 - fudge (src/mtsmd.f:474), constraints energy
// only (their forces would be removed by the constraints)
// a non-equilibrium schedule drives the lambdas (ne.cu)
static bool md_ne(const orac_gpu_ctx* ctx) { return ctx->ne.on && ctx->d_ne && ctx->variant == VAR_ALCH; }
// the work term of a level's shell: 0 M, 1 L, 2 H (+3: its reciprocal sum)
static int ne_term(int lvl) { return lvl == LM ? 0 : (lvl == LL ? 1 : 2); }

static int md_ferrf(orac_gpu_ctx* ctx, MdState& S, unsigned long long* f, bool energy) {
  const BondedDev& B = ctx->bd;
  const double* q = ctx->pme_q();
  // d/dlambda of the corrections of alchemical charges (ferrf_alchemy)
  const double* dq = (energy && ctx->variant == VAR_ALCH) ? ctx->d_dq : nullptr;
  double* edq = dq ? S.e + E_DUDL + 4 : nullptr;
  // bonds, constraints (energy only, and only when energies are wanted),
  // 1-3 pairs, 1-4 pairs: one launch, each list into its energy slots
  const int* lists[4] = {B.pbond, B.pcn, B.p13, B.p14};
  const int n[4] = {B.nb, energy ? B.ncn : 0, B.n13, B.n14};
  const double fudge[4] = {1.0, 1.0, 1.0, 1.0 - B.fudge};
  const int forces[4] = {1, 0, 1, 1};
  double* e[4] = {energy ? S.e + E_ERF : nullptr, S.e + E_ERF + 4, energy ? S.e + E_ERF + 8 : nullptr,
                  energy ? S.e + E_ERF + 12 : nullptr};
  return ferrf_launch_lists(ctx, 4, lists, n, fudge, forces, e, S.x, B.ss, q, f, dq, edq);
}

// one shell's pair forces into its level accumulator (zeroed by the
// preceding drift, or here when `zero`)
static int md_shell_pair(orac_gpu_ctx* ctx, MdState& S, char sh, int lvl, bool zero, double* e, bool energy,
                         bool no_next = false) {
  unsigned long long* f = S.ffix[lvl];
  if (zero) CK(cudaMemsetAsync(f, 0, sizeof(unsigned long long) * 3 * ctx->N, ctx->stream));
  // along a schedule force_alchemy's dwrk, U(lambda) - U(lambda0) over the
  // shell's pairs, is a work term: an energy evaluation yields it with the
  // energies, a forces-only one sums it over the alchemical pairs; either
  // way it stays pending until the M step's work sum commits it
  const bool ne = md_ne(ctx);
  double* pend = ne ? &ctx->d_ne->dwn[ne_term(lvl)] : nullptr;
  if (ne && !energy) {
    CK(cudaMemsetAsync(pend, 0, sizeof(double), ctx->stream));
    ctx->pair_dwrk = pend;
  }
  const int flags = SH_PREPPED | SH_FIXED_OUT | (energy ? SH_ENERGY : 0) | (no_next ? SH_NO_NEXT : 0);
  const int rc0 = shell_run_r(ctx, sh, ctx->sh, ctx->d_xyz, ctx->d_grp, ctx->d_mol, reinterpret_cast<double*>(f),
                              energy ? e : nullptr, nullptr, flags);
  ctx->pair_dwrk = nullptr;
  if (rc0) return rc0;
  if (ne && energy)
    CK(cudaMemcpyAsync(pend, ctx->d_xtra + 1, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  const bool dudl = energy && ctx->variant == VAR_ALCH && ctx->d_dq;
  if (dudl)  // the shell's dU/dlambda (k_variant_out)
    CK(cudaMemcpyAsync(S.e + E_DUDL + lvl, ctx->d_xtra + 4, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (energy && ctx->variant == VAR_REM)  // the shell's REM segment energy (seg_ene)
    CK(cudaMemcpyAsync(S.e + E_DUDL + lvl, ctx->d_xtra, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  return ORAC_OK;
}

// SPME and the erf corrections of the shell that carries the reciprocal
// term (mts_furier, src/mts_furier.f:71-133), into the same accumulator
static bool md_has_recip(const orac_gpu_ctx* ctx, const MdState& S, char sh) { return ctx->clewld && S.rshk == sh; }

static int md_shell_recip(orac_gpu_ctx* ctx, MdState& S, char sh, int lvl, bool energy) {
  if (!md_has_recip(ctx, S, sh)) return ORAC_OK;
  unsigned long long* f = S.ffix[lvl];
  const bool dudl = energy && ctx->variant == VAR_ALCH && ctx->d_dq;
  double recip[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) recip[i + 3 * j] = 0.5 * ctx->oc[j + 3 * i];  // src/fft_pme.f:47-51
  int slot = -1;
  if (int rc = prof_begin(ctx, &slot, PROF_PME)) return rc;
  // along a schedule the transformed grid of chrgec is kept for the work
  float2* keep = md_ne(ctx) ? ctx->pme.cgsave : nullptr;
  if (int rc = pme_run(ctx, ctx->N, S.x, ctx->pme_q(), recip, ctx->volume, ctx->alphal, nullptr, S.e + 24, nullptr,
                       nullptr, f, dudl ? ctx->d_dq : nullptr, dudl ? S.e + E_DUDL + 3 : nullptr, keep))
    return rc;
  if (int rc = prof_end(ctx, slot)) return rc;
  if (!md_ne(ctx)) return md_ferrf(ctx, S, f, energy);
  // along a schedule: mts_furier_alchemy's dwrk (src/mts_furier_alchemy.f:
  // 112-186), the SPME sum, erf corrections and self term of chrgec minus
  // those of chrge0; a second SPME, of chrgec - chrge0 against the kept
  // grid of chrgec, gives the SPME difference (energy only)
  const BondedDev& B = ctx->bd;
  const int* lists[4] = {B.pbond, B.pcn, B.p13, B.p14};
  const int n[4] = {B.nb, B.ncn, B.n13, B.n14};
  const double fudge[4] = {1.0, 1.0, 1.0, 1.0 - B.fudge};
  const int forces[4] = {1, 0, 1, 1};
  double* eq[4] = {S.e + E_NEQ, S.e + E_NEQ + 4, S.e + E_NEQ + 8, S.e + E_NEQ + 12};
  double* e0[4] = {S.e + E_NEQ0, S.e + E_NEQ0 + 4, S.e + E_NEQ0 + 8, S.e + E_NEQ0 + 12};
  CK(cudaMemsetAsync(S.e + E_NEQ, 0, sizeof(double) * 32, ctx->stream));
  if (int rc = ferrf_launch_lists(ctx, 4, lists, n, fudge, forces, eq, S.x, B.ss, ctx->d_qc, f, nullptr, nullptr))
    return rc;
  if (energy)  // the energy record's erf corrections
    CK(cudaMemcpyAsync(S.e + E_ERF, S.e + E_NEQ, sizeof(double) * 16, cudaMemcpyDeviceToDevice, ctx->stream));
  if (int rc = pme_run(ctx, ctx->N, S.x, ctx->d_ne_dq, recip, ctx->volume, ctx->alphal, nullptr, S.e + E_NE0,
                       nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, ctx->pme.cgsave))
    return rc;
  if (int rc = ferrf_launch_lists(ctx, 4, lists, n, fudge, forces, e0, S.x, B.ss, ctx->d_q0, nullptr, nullptr,
                                  nullptr))
    return rc;
  return ne_recip_launch(ctx, S.e + E_NE0, S.e + E_NEQ, S.e + E_NEQ0, 3 + ne_term(lvl));
}

static int md_forces_shell(orac_gpu_ctx* ctx, MdState& S, char sh, int lvl, bool zero, double* e, bool energy) {
  if (int rc = md_shell_pair(ctx, S, sh, lvl, zero, e, energy)) return rc;
  return md_shell_recip(ctx, S, sh, lvl, energy);
}

// Fork and join of the step's second stream; launches between them go to
// the side stream while the shell pair kernels run on the context's own.
struct SideStream {
  orac_gpu_ctx* ctx;
  cudaStream_t side;
  cudaEvent_t ev_fork, ev_join;
  int fork() {
    CK(cudaEventRecord(ev_fork, ctx->stream));
    CK(cudaStreamWaitEvent(side, ev_fork, 0));
    return ORAC_OK;
  }
  int join() {
    CK(cudaEventRecord(ev_join, side));
    CK(cudaStreamWaitEvent(ctx->stream, ev_join, 0));
    return ORAC_OK;
  }
  template <typename F>
  int run(F&& fn) {  // every launcher uses ctx->stream: point it at the side stream meanwhile
    cudaStream_t own = ctx->stream;
    ctx->stream = side;
    const int rc = fn();
    ctx->stream = own;
    return rc;
  }
};

// mts_intra_n0 / mts_intra_n1 into their level accumulators
// 1-4 and intra-group pairs of the N1 level (fnb14, fnbgrp)
// ORAC's intra-alchemical corrections apply with alchemy and Ewald
// (src/mts_intra_n1.f:81-85, src/mtsmd.f:3035-3041)
static bool md_alch_intra(const orac_gpu_ctx* ctx) {
  return ctx->variant == VAR_ALCH && ctx->clewld && ctx->d_lam4;
}

// The N1 level's pair terms (fnb14 -- fnb14_alchemy with alchemy and Ewald,
// src/mts_intra_n1.f:81-85 -- and fnbgrp) in one launch, and, when the step
// ends an M step too (with_m), ferrf_alchemy_add over listqq into the M
// accumulator (src/mtsmd.f:3035-3041): every M step is an N1 step, so the
// correction costs no launch of its own.
static int md_pairs_n1(orac_gpu_ctx* ctx, MdState& S, bool energy, bool with_m = false) {
  const BondedDev& B = ctx->bd;
  SmallSpec sp[3];
  int n = 0;
  const int coul = ctx->clewld ? 1 : 0;
  const bool alch = md_alch_intra(ctx);
  const bool ne = md_ne(ctx);
  if (B.have_pairs && B.n14 > 0) {
    sp[n++] = {alch ? 3 : 0, S.x, B.p14, B.t14, B.n14, B.e1412, B.e146, B.fudge, B.lj_fudge, coul,
               energy ? S.e + E_14 : nullptr, B.ss, ctx->d_aqd, S.ffix[LN1],
               (alch && energy) ? S.e + E_DUDL + 5 : nullptr};
    if (ne && alch) {  // fnb14_alchemy's dwrk of this evaluation is dwrk14 (src/mtsmd.f:2903)
      CK(cudaMemsetAsync(&ctx->d_ne->dwn[7], 0, sizeof(double), ctx->stream));
      sp[n - 1].work = &ctx->d_ne->dwn[7];
    }
  }
  if (B.have_pairs && B.ningrp > 0)
    sp[n++] = {1, S.x, B.pgrp, B.nbt, B.ningrp, B.e12, B.e6, 1.0, 1.0, coul, energy ? S.e + E_GRP : nullptr, B.ss,
               ctx->d_aqd, S.ffix[LN1], nullptr};
  if (with_m && alch && !ne) {
    if (ctx->nlistqq < 0)
      if (int rc = alch_listqq_build(ctx)) return rc;
    if (ctx->nlistqq > 0)
      sp[n++] = {4, S.x, ctx->d_listqq, nullptr, ctx->nlistqq, nullptr, nullptr, 1.0, 1.0, 1,
                 energy ? S.e + E_AQQ : nullptr, B.ss, ctx->d_aqd, S.ffix[LM], energy ? S.e + E_DUDL + 6 : nullptr};
  }
  return small_launch_set(ctx, n, sp);
}

// ferrf_alchemy_add on an M step of a system without N1 pair terms
static int md_alch_m(orac_gpu_ctx* ctx, MdState& S, bool energy) {
  if (!md_alch_intra(ctx) || (S.has_n1 && !md_ne(ctx))) return ORAC_OK;
  if (md_ne(ctx)) {  // ferrf_alchemy_add's dwrk is dwrk_al (src/mtsmd.f:3035-3041)
    if (ctx->nlistqq < 0)
      if (int rc = alch_listqq_build(ctx)) return rc;
    if (ctx->nlistqq <= 0) return ORAC_OK;
    SmallSpec sp = {4, S.x, ctx->d_listqq, nullptr, ctx->nlistqq, nullptr, nullptr, 1.0, 1.0, 1,
                    energy ? S.e + E_AQQ : nullptr, ctx->bd.ss, ctx->d_aqd, S.ffix[LM], nullptr,
                    &ctx->d_ne->dwn[6]};
    return small_launch_set(ctx, 1, &sp);
  }
  if (ctx->nlistqq < 0)
    if (int rc = alch_listqq_build(ctx)) return rc;
  return alch_intra_launch(ctx, 4, S.x, S.ffix[LM], energy ? S.e + E_AQQ : nullptr,
                           energy ? S.e + E_DUDL + 6 : nullptr);
}

// the bonded terms of the N0 level (stretching, bending, impropers) and/or
// the N1 level (proper torsions) in one launch, each into its accumulator
static int md_bonded(orac_gpu_ctx* ctx, MdState& S, bool n0, bool n1, bool energy) {
  const int mask = (n0 ? BK_BOND | BK_BEND | BK_ITORS : 0) | (n1 ? BK_TORS : 0);
  if (!mask) return ORAC_OK;
  int slot = -1;
  if (int rc = prof_begin(ctx, &slot, PROF_BONDED)) return rc;
  if (int rc = bonded_launch(ctx, mask, S.x, nullptr, S.ffix[LN0], energy ? S.e + E_BOND : nullptr, S.ffix[LN1]))
    return rc;
  return prof_end(ctx, slot);
}

static int md_forces_intra(orac_gpu_ctx* ctx, MdState& S, int lvl, bool energy) {
  if (int rc = md_bonded(ctx, S, lvl == LN0, lvl == LN1, energy)) return rc;
  return lvl == LN1 ? md_pairs_n1(ctx, S, energy, true) : ORAC_OK;
}

static int md_phony(orac_gpu_ctx* ctx, const ShellRadii& r, char sh) {
  return shell_run_r(ctx, sh, r, ctx->d_xyz, ctx->d_grp, ctx->d_mol, nullptr, nullptr, nullptr,
                     SH_PREPPED | SH_FIXED_OUT);
}

static int md_list_update(orac_gpu_ctx* ctx, MdState& S) {
  const ShellRadii r = ctx->sh;
  if (int rc = list_build_cells_async(ctx, r.rcuth + r.rtolh + r.rneih, &ctx->lists[0], S.flag)) return rc;
  ShellRadii r1 = r;
  r1.rcuth = r.rcutl;
  r1.rtolh = 0.0;
  if (int rc = md_phony(ctx, r1, 'h')) return rc;
  ShellRadii r2 = r1;
  r2.rcutl = r.rcutm;
  r2.rtoll = 0.0;
  return md_phony(ctx, r2, 'l');
}

// One outer step as a sequence of K = lrespa mrespa n1respa n0respa drifts
// of tn0.  Level l (periods pN0 = 1, pN1 = n0respa, pM = pN1 n1respa, pL =
// pM mrespa, pH = K drifts) ends its inner step after drift k when
// (k+1) % p == 0: its forces are evaluated there, and its end half kick
// and the next step's start half kick (correc + rattle_correc twice at the
// same instant) are applied together before the next drift.  The start half
// kicks of the outer step go before the first drift; all end half kicks come
// after the last force evaluation.  The N0 start half kick is verlet's,
// without RATTLE (src/verlet.f), as in ORAC's n0 loop
// (src/mtsmd.f:2641-2930).
static int md_step(orac_gpu_ctx* ctx, MdState& S, bool update, bool energy) {
  if (update)
    if (int rc = md_list_update(ctx, S)) return rc;
  if (energy) CK(cudaMemsetAsync(S.e + E_BOND, 0, sizeof(double) * (E_N - E_BOND), ctx->stream));
  const int n0 = S.n0respa, n1 = S.n1respa;
  const int per[NLV] = {S.lrespa * S.mrespa * n1 * n0, S.mrespa * n1 * n0, n1 * n0, n0, 1};
  const int K = per[LH];
  SideStream sd{ctx, S.side, S.ev_fork, S.ev_join};
  SideStream sd2{ctx, S.side2, S.ev_fork2, S.ev_join2};
  double dt[NLV];
  dt[LH] = S.dth;
  dt[LL] = dt[LH] / S.lrespa;
  dt[LM] = dt[LL] / S.mrespa;
  dt[LN1] = dt[LM] / n1;
  dt[LN0] = dt[LN1] / n0;
  for (int k = 0; k < K; k++) {
    double c[NLV] = {0, 0, 0, 0, 0};
    if (k == 0) {
      for (int l = 0; l < LN0; l++) c[l] = 0.5 * dt[l];
    } else {
      c[LN0] = 0.5 * dt[LN0];  // end half kick of the last N0 step (the start one is verlet's)
      for (int l = LL; l < LN0; l++)
        if (k % per[l] == 0) c[l] = dt[l];
    }
    const bool tstart = S.th && k % per[LM] == 0;
    if (tstart) {
      // an M step starts: the end of the previous one (its N0 and N1 end
      // half kicks and the M sandwich, K1), the L kicks at an L boundary
      // (the H and L start kicks at the step's start), K2; the drift then
      // applies the start sandwich and the N1 start half kick
      const bool first = k == 0;
      if (int rc = md_thermo(ctx, S, !first, true, first ? 0.0 : 0.5 * dt[LN0], first ? 0.0 : 0.5 * dt[LN1],
                             0.5 * dt[LM], c[LL], c[LH]))
        return rc;
      for (int l = 0; l < NLV; l++) c[l] = l == LN1 ? 0.5 * dt[LN1] : 0.0;
    }
    int zmask = 0;
    for (int l = 0; l < NLV; l++)
      if ((k + 1) % per[l] == 0) zmask |= 1 << l;
    if (int rc = md_drift(ctx, S, dt[LN0], c, zmask, (k + 1) % per[LM] == 0, tstart)) return rc;
    const bool last = k == K - 1;
    const bool e_now = energy && last;
    const bool due_n1 = S.has_n1 && (k + 1) % per[LN1] == 0;
    const bool due_m = (k + 1) % per[LM] == 0, due_l = (k + 1) % per[LL] == 0;
    // intramolecular levels and SPME beside the shell pair kernels: each
    // adds into its own level accumulator (SPME into the pair kernel's, by
    // exact fixed-point atomics), and all are joined before the next drift
    // the last drift also ends the H step: the H shell (after the L shell,
    // whose list it rewrites) and its reciprocal sum join the same fork, so
    // the H pair kernel overlaps the L level's SPME
    const bool side = S.has_n0 || due_n1 || (due_m && md_has_recip(ctx, S, 'm')) ||
                      (due_l && md_has_recip(ctx, S, 'l')) || (last && md_has_recip(ctx, S, 'h'));
    // along a schedule the M step's order is ORAC's: the N1 level's pairs
    // with the old lambdas, the lambda update, then every shell and
    // reciprocal sum with the new ones (src/mtsmd.f:2900-3060)
    const bool ne_m = md_ne(ctx) && due_m;
    if (ne_m) {
      if (due_n1)
        if (int rc = md_pairs_n1(ctx, S, e_now, false)) return rc;
      if (int rc = ne_lambda_launch(ctx, per[LM])) return rc;
    }
    if (side) {
      if (int rc = sd.fork()) return rc;
      if (int rc = sd.run([&]() -> int {
            if (int r2 = md_bonded(ctx, S, S.has_n0, due_n1, e_now)) return r2;
            if (due_m)
              if (int r2 = md_shell_recip(ctx, S, 'm', LM, e_now)) return r2;
            if (due_l)
              if (int r2 = md_shell_recip(ctx, S, 'l', LL, e_now)) return r2;
            if (last)
              if (int r2 = md_shell_recip(ctx, S, 'h', LH, energy)) return r2;
            return ORAC_OK;
          }))
        return rc;
    }
    // the last drift of a step without energies: the L shell (its M list
    // is rebuilt below anyway, so it writes none) and then the H shell (which
    // rewrites the L list) on a third stream beside the M shell; the M list
    // is rebuilt from the new L list once both are done.  The shells of an
    // energy step share the energy accumulators and run one after another.
    const bool split3 = last && !energy;
    if (split3) {
      if (int rc = sd2.fork()) return rc;
      if (int rc = sd2.run([&]() -> int {
            if (int r2 = md_shell_pair(ctx, S, 'l', LL, false, S.e + 8, false, true)) return r2;
            return md_shell_pair(ctx, S, 'h', LH, false, S.e + 16, false);
          }))
        return rc;
    }
    if (due_m) {
      if (int rc = md_shell_pair(ctx, S, 'm', LM, false, S.e, e_now)) return rc;
      if (int rc = md_alch_m(ctx, S, e_now)) return rc;  // only without N1 pairs (else with them)
    }
    if (due_l && !split3)
      if (int rc = md_shell_pair(ctx, S, 'l', LL, false, S.e + 8, e_now)) return rc;
    if (last) {
      if (split3) {
        if (int rc = sd2.join()) return rc;
      } else if (int rc = md_shell_pair(ctx, S, 'h', LH, false, S.e + 16, energy)) {
        return rc;
      }
      // the M list again from the new L list (src/mtsmd.f:3287-3295)
      ShellRadii r = ctx->sh;
      r.rcutl = r.rcutm;
      if (int rc = md_phony(ctx, r, 'l')) return rc;
    }
    // the N1 level's pair terms beside the bonded kernel on the side stream
    if (due_n1 && !ne_m)
      if (int rc = md_pairs_n1(ctx, S, e_now, due_m)) return rc;
    if (side)
      if (int rc = sd.join()) return rc;
    if (ne_m) {
      // the M step's work, then the terms evaluated here become the held
      // ones: M shell, listqq, 1-4, and the L shell and the reciprocal sums
      // of the levels evaluated at this step
      int commit = 1 | (1 << 6) | (1 << 7);
      if (due_l) commit |= 1 << 1;
      if (last) commit |= 1 << 2;
      if (md_has_recip(ctx, S, 'm')) commit |= 1 << 3;
      if (due_l && md_has_recip(ctx, S, 'l')) commit |= 1 << 4;
      if (last && md_has_recip(ctx, S, 'h')) commit |= 1 << 5;
      if (int rc = ne_sum_launch(ctx, commit)) return rc;
    }
  }
  if (S.th) {
    // the last M step's end (K1) and the end half kicks of L and H
    if (int rc = md_thermo(ctx, S, true, false, 0.5 * dt[LN0], 0.5 * dt[LN1], 0.5 * dt[LM], 0.5 * dt[LL],
                           0.5 * dt[LH]))
      return rc;
  } else {
    double c[NLV];
    for (int l = 0; l < NLV; l++) c[l] = 0.5 * dt[l];
    if (int rc = md_kick(ctx, S, c)) return rc;
  }
  if (energy) {
    CK(cudaMemsetAsync(S.e + 40, 0, sizeof(double), ctx->stream));
    orac_launch(k_ekin, 64, 256, 0, ctx->stream, ctx->N, S.v, S.invm, S.e + 40);
    CKL();
    const int var = md_ne(ctx) ? 3 : ((ctx->variant == VAR_ALCH && ctx->d_dq) ? 2 : (ctx->variant == VAR_REM ? 1 : 0));
    orac_launch(k_record, 1, 32, 0, ctx->stream, S.e, S.flag, S.econst, ctx->self_dudl, var, S.rec, S.rec_cap,
                S.rec_n, (const NeDev*)ctx->d_ne, (const ThermoDev*)S.th);
    CKL();
  }
  return ORAC_OK;
}

static int md_run_impl(orac_gpu_ctx* ctx, int nsteps, int energy_every, double* rec, bool async);

// THERMOS (src/find_thermos.f, src/cov_thermos.f): degrees of freedom 3 per
// molecule (centres of mass), 3 per atom less 3 per molecule less the
// constraints (solute; solvent); Q = 2 ndf k T / (2 pi c nu)^2, zero for a
// class without atoms or with one degree of freedom
static int thermo_setup(orac_gpu_ctx* ctx, MdState& S, const std::vector<int>& ma0, const std::vector<int>& mna,
                        const std::vector<char>& small, int ncnst, const int* cnst, double tm) {
  if (S.nbig)
    return ctx_fail(ctx, ORAC_ERR_PARAM, "thermostats with constraint sets solved iteratively (more than %d atoms "
                                         "or %d constraints joined) are not supported", SMA, SMC);
  const int N = ctx->N, P = ctx->P;
  std::vector<int> cls(N), abm(N, -1);
  std::vector<int4> br;
  std::vector<double> bm;
  int nat[3] = {0, 0, 0}, nmol[3] = {0, 0, 0}, ncn[3] = {0, 0, 0};
  for (int a = 0; a < N; a++) {
    cls[a] = ctx->h_ss[a] == 1 ? 1 : 2;
    nat[cls[a]]++;
  }
  for (int p = 0; p < P; p++) {
    if (mna[p] <= 0) continue;
    nmol[cls[ma0[p]]]++;
    if (small[p]) continue;
    double m = 0.0;
    const int b = (int)bm.size();
    for (int a = ma0[p]; a < ma0[p] + mna[p]; a++) {
      abm[a] = b;
      m += ctx->h_mass[a];
    }
    for (int a = ma0[p]; a < ma0[p] + mna[p]; a += TH_CHUNK)
      br.push_back(make_int4(b, a, std::min(TH_CHUNK, ma0[p] + mna[p] - a), 0));
    bm.push_back(m);
  }
  for (int k = 0; k < ncnst; k++) ncn[cls[cnst[2 * k] - 1]]++;
  int ndf[3] = {3 * P, 3 * nat[1] - 3 * nmol[1] - ncn[1], 3 * nat[2] - 3 * nmol[2] - ncn[2]};
  const double avogad = 6.022140857e23, boltz = 1.38064852e-23;  // src/setuns.f:37-38
  const double unitm = 1.0 / (avogad * 1000.0), unitl = 1.0e-10, unite = unitm * (unitl / 1.0e-15) * (unitl / 1.0e-15);
  const double c = 2.0 * 3.14159265358979323846 * 2.997925e10;
  ThermoDev T;
  memset(&T, 0, sizeof(T));
  for (int k = 0; k < 3; k++) {
    const bool exist = k == 0 || nat[k] > 0;
    const double om = ctx->thermo.nu[k] * c;
    T.q[k] = exist ? 2.0 * ndf[k] * boltz * ctx->thermo.temp / (om * om) / (unitm * unitl * unitl) : 0.0;
    if (ndf[k] == 1) T.q[k] = 0.0;
    T.ndfkt[k] = ndf[k] * boltz * ctx->thermo.temp / unite;
    T.s[k] = 1.0;
    S.th_ndf[k] = ndf[k];
  }
  T.tm = tm;
  T.tm4 = 0.25 * tm;
  S.th_tm = tm;
  S.nbm = (int)bm.size();
  S.nchunk = (int)br.size();
  S.th_blocks = (S.nsm + S.nfree + S.nbm + TH_BLOCK - 1) / TH_BLOCK;
  if (dev_alloc(ctx, &S.th, 1) || dev_alloc(ctx, &S.tpart, 6 * (size_t)S.th_blocks) || dev_alloc(ctx, &S.tcls, N) ||
      dev_alloc(ctx, &S.abm, N))
    return ORAC_ERR_CUDA;
  CK(cudaMemcpy(S.th, &T, sizeof(T), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(S.tcls, cls.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(S.abm, abm.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  if (S.nbm) {
    if (dev_alloc(ctx, &S.bchunk, S.nchunk) || dev_alloc(ctx, &S.bmass, S.nbm) ||
        dev_alloc(ctx, &S.msum, (size_t)TH_NS * S.nbm) || dev_alloc(ctx, &S.vcur, 3 * (size_t)S.nbm))
      return ORAC_ERR_CUDA;
    CK(cudaMemcpy(S.bchunk, br.data(), sizeof(int4) * S.nchunk, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(S.bmass, bm.data(), sizeof(double) * S.nbm, cudaMemcpyHostToDevice));
  }
  return ORAC_OK;
}

// The six N-double arrays of a state transfer as few copies as possible:
// arrays that follow each other in memory on both sides go as one copy.
static int copy_runs(orac_gpu_ctx* ctx, double* const dst[6], const double* const src[6], cudaMemcpyKind kind) {
  const size_t N = (size_t)ctx->N;
  for (int k = 0; k < 6;) {
    int e = k + 1;
    while (e < 6 && dst[e] == dst[e - 1] + N && src[e] == src[e - 1] + N) e++;
    CK(cudaMemcpyAsync(dst[k], src[k], (size_t)(e - k) * N * sizeof(double), kind, ctx->stream));
    k = e;
  }
  return ORAC_OK;
}

extern "C" {

int orac_gpu_md_setup(orac_gpu_ctx* ctx, const double* x, const double* y, const double* z, const double* vx,
                      const double* vy, const double* vz, const int* cnst, const double* dss, int ncnst,
                      double dt_h, int lrespa, int mrespa, int n1respa, int n0respa, int nupdte, char rshk,
                      double econst) {
  if (!ctx || !ctx->have_topo || !ctx->have_box || !ctx->have_shells || !ctx->have_ewald)
    return ctx ? ctx_fail(ctx, ORAC_ERR_STATE, "md_setup before topology/box/shells/ewald") : ORAC_ERR_PARAM;
  if (ctx->ncx <= 0) return ctx_fail(ctx, ORAC_ERR_STATE, "md needs LINKED_CELL");
  if (dt_h <= 0 || lrespa < 1 || mrespa < 1 || n1respa < 1 || n0respa < 1 || nupdte < 1)
    return ctx_fail(ctx, ORAC_ERR_PARAM, "bad r-RESPA schedule");
  CK(cudaSetDevice(ctx->device));
  md_destroy(ctx);
  MdState& S = *md_of(ctx);
  const int N = ctx->N, P = ctx->P, G = ctx->G;
  S.N = N;
  CK(cudaStreamCreateWithFlags(&S.side, cudaStreamNonBlocking));
  CK(cudaMallocHost((void**)&S.h_flag, sizeof(int)));
  CK(cudaEventCreateWithFlags(&S.ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&S.ev_join, cudaEventDisableTiming));
  CK(cudaStreamCreateWithFlags(&S.side2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&S.ev_fork2, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&S.ev_join2, cudaEventDisableTiming));
  // positions and velocities in one allocation, back to back: a state
  // transfer to or from a packed host buffer is one copy each way
  if (dev_alloc(ctx, &S.x, 6 * (size_t)N) ||
      dev_alloc(ctx, &S.xo, 3 * (size_t)N) || dev_alloc(ctx, &S.ffix[0], 3 * (size_t)N) ||
      dev_alloc(ctx, &S.ffix[1], 3 * (size_t)N) || dev_alloc(ctx, &S.ffix[2], 3 * (size_t)N) ||
      dev_alloc(ctx, &S.invm, N) || dev_alloc(ctx, &S.pm, N) || dev_alloc(ctx, &S.e, E_ALL) || dev_alloc(ctx, &S.rec, (size_t)ORAC_MD_REC * MD_REC_CAP) ||
      dev_alloc(ctx, &S.rec_n, 1) ||
      dev_alloc(ctx, &S.flag, 4))
    return ORAC_ERR_CUDA;
  S.v = S.x + 3 * (size_t)N;
  {
    // intramolecular levels (mts_intra_n0 / mts_intra_n1) when the topology has terms for them
    const BondedDev& B = ctx->bd;
    S.has_n0 = B.nb + B.nbend + B.nit > 0;
    S.has_n1 = B.nt > 0 || (B.have_pairs && B.n14 + B.ningrp > 0);
    if ((S.has_n1 && dev_alloc(ctx, &S.ffix[LN1], 3 * (size_t)N)) ||
        (S.has_n0 && dev_alloc(ctx, &S.ffix[LN0], 3 * (size_t)N)))
      return ORAC_ERR_CUDA;
    CK(cudaMemset(S.e, 0, sizeof(double) * E_ALL));
    CK(cudaMemset(S.rec_n, 0, sizeof(unsigned long long)));
    S.rec_cap = MD_REC_CAP;
  }
  if (int rc = bonded_set_constraints(ctx, cnst, ncnst)) return rc;
  const double* src[2][3] = {{x, y, z}, {vx, vy, vz}};
  double* dst[2] = {S.x, S.v};
  for (int k = 0; k < 2; k++)
    for (int d = 0; d < 3; d++)
      CK(cudaMemcpy(dst[k] + (size_t)d * N, src[k][d], sizeof(double) * N, cudaMemcpyHostToDevice));
  std::vector<double> im(N), pm(N);
  for (int a = 0; a < N; a++) im[a] = 1.0 / ctx->h_mass[a];
  for (int g = 0; g < G; g++) {
    double mt = 0;
    for (int a = ctx->h_gfirst[g]; a < ctx->h_gfirst[g] + ctx->h_gn[g]; a++) mt += ctx->h_mass[a];
    for (int a = ctx->h_gfirst[g]; a < ctx->h_gfirst[g] + ctx->h_gn[g]; a++) pm[a] = ctx->h_mass[a] / mt;
  }
  CK(cudaMemcpy(S.invm, im.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(S.pm, pm.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  // molecule atom ranges (contiguous) and group ranges
  std::vector<int> ma0(P, -1), mna(P, 0), mg0(P, -1), mng(P, 0);
  for (int a = 0; a < N; a++) {
    const int p = ctx->h_amol[a];
    if (a > 0 && ctx->h_amol[a] < ctx->h_amol[a - 1])
      return ctx_fail(ctx, ORAC_ERR_PARAM, "molecules must be contiguous");
    if (ma0[p] < 0) ma0[p] = a;
    mna[p]++;
  }
  for (int g = 0; g < G; g++) {
    const int p = ctx->h_gmol[g];
    if (mg0[p] < 0) mg0[p] = g;
    mng[p]++;
  }
  std::vector<std::vector<int>> bym(P);
  for (int k = 0; k < ncnst; k++) {
    const int a = cnst[2 * k] - 1, b = cnst[2 * k + 1] - 1;
    if (a < 0 || a >= N || b < 0 || b >= N || ctx->h_amol[a] != ctx->h_amol[b] || dss[k] <= 0)
      return ctx_fail(ctx, ORAC_ERR_PARAM, "constraint %d", k + 1);
    bym[ctx->h_amol[a]].push_back(k);
  }
  std::vector<int4> sm;
  std::vector<int2> smg, cloc, bcab;
  std::vector<double> cd, bd;
  std::vector<int> bst = {0}, fa, fg;
  std::vector<char> small(P, 0), in_cluster(N, 0);
  std::vector<int> sm_atoms;
  for (int p = 0; p < P; p++) {
    const int nc = (int)bym[p].size();
    if (nc > 0 && nc <= SMC && mna[p] <= SMA) {
      small[p] = 1;
      // a rigid triangle (3 atoms, pairs 01, 02, 12) gets the closed-form solver
      int slot[3] = {-1, -1, -1};
      if (nc == 3 && mna[p] == 3)
        for (int k : bym[p]) {
          int a = cnst[2 * k] - 1 - ma0[p], b = cnst[2 * k + 1] - 1 - ma0[p];
          if (a > b) std::swap(a, b);
          const int s = (a == 0 && b == 1) ? 0 : (a == 0 && b == 2) ? 1 : (a == 1 && b == 2) ? 2 : -1;
          if (s >= 0) slot[s] = k;
        }
      const bool tri = slot[0] >= 0 && slot[1] >= 0 && slot[2] >= 0;
      sm.push_back(make_int4(ma0[p], mna[p], (int)cloc.size(), nc | (tri ? MOL3 : 0)));
      smg.push_back(make_int2(mg0[p], mng[p]));
      if (tri) {
        const int2 pr[3] = {make_int2(0, 1), make_int2(0, 2), make_int2(1, 2)};
        for (int q = 0; q < 3; q++) {
          cloc.push_back(pr[q]);
          cd.push_back(dss[slot[q]]);
        }
      } else {
        for (int k : bym[p]) {
          cloc.push_back(make_int2(cnst[2 * k] - 1 - ma0[p], cnst[2 * k + 1] - 1 - ma0[p]));
          cd.push_back(dss[k]);
        }
      }
    } else if (nc > 0) {
      // a large molecule: its constraints split into connected clusters
      // (a heavy atom with its hydrogens, typically); those of at most SMA
      // atoms and SMC constraints are solved like small molecules, the rest
      // by the iterative SHAKE/RATTLE of large molecules, one unit each.
      // Clusters share no atom, so this is the same constrained solution.
      std::vector<int> par(mna[p]);
      for (int q = 0; q < mna[p]; q++) par[q] = q;
      auto find = [&](int q) {
        while (par[q] != q) q = par[q] = par[par[q]];
        return q;
      };
      for (int k : bym[p]) {
        const int a = find(cnst[2 * k] - 1 - ma0[p]), b = find(cnst[2 * k + 1] - 1 - ma0[p]);
        if (a != b) par[std::max(a, b)] = std::min(a, b);
      }
      std::vector<std::vector<int>> comp_c(mna[p]);
      for (int k : bym[p]) comp_c[find(cnst[2 * k] - 1 - ma0[p])].push_back(k);
      for (int r = 0; r < mna[p]; r++) {
        const std::vector<int>& ks = comp_c[r];
        if (ks.empty()) continue;
        std::vector<int> atoms;
        for (int k : ks)
          for (int e = 0; e < 2; e++) atoms.push_back(cnst[2 * k + e] - 1);
        std::sort(atoms.begin(), atoms.end());
        atoms.erase(std::unique(atoms.begin(), atoms.end()), atoms.end());
        if ((int)atoms.size() <= SMA && (int)ks.size() <= SMC) {
          auto loc = [&](int a) { return (int)(std::lower_bound(atoms.begin(), atoms.end(), a) - atoms.begin()); };
          int slot[3] = {-1, -1, -1};
          if (ks.size() == 3 && atoms.size() == 3)
            for (int k : ks) {
              int a = loc(cnst[2 * k] - 1), b = loc(cnst[2 * k + 1] - 1);
              if (a > b) std::swap(a, b);
              const int sl = (a == 0 && b == 1) ? 0 : (a == 0 && b == 2) ? 1 : (a == 1 && b == 2) ? 2 : -1;
              if (sl >= 0) slot[sl] = k;
            }
          const bool tri = slot[0] >= 0 && slot[1] >= 0 && slot[2] >= 0;
          // a star: one atom in every constraint and one constraint per
          // other atom; listed centre first, constraint k to atom k + 1
          int centre = -1;
          if (!tri && (int)ks.size() == (int)atoms.size() - 1)
            for (int a : atoms) {
              bool all = true;
              for (int k : ks) all = all && (cnst[2 * k] - 1 == a || cnst[2 * k + 1] - 1 == a);
              if (all) {
                centre = a;
                break;
              }
            }
          if (centre >= 0) {
            atoms.clear();
            atoms.push_back(centre);
            for (int k : ks) atoms.push_back(cnst[2 * k] - 1 == centre ? cnst[2 * k + 1] - 1 : cnst[2 * k] - 1);
          }
          sm.push_back(make_int4((int)sm_atoms.size(), (int)atoms.size(), (int)cloc.size(),
                                 (int)ks.size() | CLUSTER | (tri ? MOL3 : 0) | (centre >= 0 ? STAR : 0)));
          smg.push_back(make_int2(0, 0));
          for (int a : atoms) {
            sm_atoms.push_back(a);
            in_cluster[a] = 1;
          }
          if (centre >= 0) {
            for (int q = 0; q < (int)ks.size(); q++) {
              cloc.push_back(make_int2(0, q + 1));
              cd.push_back(dss[ks[q]]);
            }
          } else if (tri) {
            const int2 pr[3] = {make_int2(0, 1), make_int2(0, 2), make_int2(1, 2)};
            for (int q = 0; q < 3; q++) {
              cloc.push_back(pr[q]);
              cd.push_back(dss[slot[q]]);
            }
          } else {
            for (int k : ks) {
              cloc.push_back(make_int2(loc(cnst[2 * k] - 1), loc(cnst[2 * k + 1] - 1)));
              cd.push_back(dss[k]);
            }
          }
        } else {
          for (int k : ks) {
            bcab.push_back(make_int2(cnst[2 * k] - 1, cnst[2 * k + 1] - 1));
            bd.push_back(dss[k]);
          }
          bst.push_back((int)bcab.size());
        }
      }
    }
  }
  // molecules outside the small ones: unconstrained (drifted by group) or
  // large constrained (drifted by atom, centred after their SHAKE)
  std::vector<int> dg, da;
  // (atoms of constraint clusters move with their cluster)
  for (int a = 0; a < N; a++)
    if (!small[ctx->h_amol[a]] && !in_cluster[a]) {
      fa.push_back(a);
      if (!bym[ctx->h_amol[a]].empty()) da.push_back(a);
    }
  for (int g = 0; g < G; g++)
    if (!small[ctx->h_gmol[g]]) (bym[ctx->h_gmol[g]].empty() ? dg : fg).push_back(g);
  // small molecules without intramolecular-level terms skip the N1 and N0
  // accumulators, which stay zero for their atoms
  {
    const bool hb = (int)ctx->h_intra_b.size() == N, hp = (int)ctx->h_intra_p.size() == N;
    for (auto& m : sm) {
      bool any = false;
      for (int q = 0; q < m.y; q++) {
        const int a = (m.w & CLUSTER) ? sm_atoms[m.x + q] : m.x + q;
        any = any || (hb && ctx->h_intra_b[a]) || (hp && ctx->h_intra_p[a]);
      }
      if (!any) m.w |= NOINTRA;
    }
  }
  S.nsm = (int)sm.size();
  S.nfree = (int)fa.size();
  S.nfreeg = (int)fg.size();
  S.ndg = (int)dg.size();
  S.nda = (int)da.size();
  S.nbig = (int)bst.size() - 1;
#define UPV(dst, vec)                                                                                        \
  if (!vec.empty()) {                                                                                        \
    if (dev_alloc(ctx, &dst, vec.size())) return ORAC_ERR_CUDA;                                            \
    CK(cudaMemcpy(dst, vec.data(), sizeof(vec[0]) * vec.size(), cudaMemcpyHostToDevice));                  \
  }
  UPV(S.sm, sm);
  UPV(S.smg, smg);
  UPV(S.cloc, cloc);
  UPV(S.cdss, cd);
  UPV(S.free_atoms, fa);
  UPV(S.free_groups, fg);
  UPV(S.drift_groups, dg);
  UPV(S.drift_atoms, da);
  UPV(S.sm_atoms, sm_atoms);
  if (S.nbig) {
    UPV(S.bstart, bst);
    UPV(S.bcab, bcab);
    UPV(S.bdss, bd);
  }
#undef UPV
  if (ctx->thermo.on)
    if (int rc = thermo_setup(ctx, S, ma0, mna, small, ncnst, cnst, dt_h / lrespa / mrespa)) return rc;
  S.dth = dt_h;
  S.lrespa = lrespa;
  S.mrespa = mrespa;
  S.n1respa = n1respa;
  S.n0respa = n0respa;
  S.nupdte = nupdte;
  S.rshk = rshk;
  S.econst = econst;
  S.step = 0;
  CK(cudaMemset(S.flag, 0, sizeof(int)));
  // positions -> scaled frame, group centres, pair-kernel inputs (a drift of
  // zero length); then the first list build with host synchronisation (it
  // sizes the list capacity with 30% headroom for in-graph rebuilds) and the
  // first forces (src/mtsmd.f:1986-2152)
  if (int rc = md_drift(ctx, S, 0.0, nullptr, 0)) return rc;
  const ShellRadii r = ctx->sh;
  const double rc_h = r.rcuth + r.rtolh + r.rneih;
  if (int rc = list_prepare_stencil(ctx, rc_h)) return rc;
  if (int rc = list_build_cells(ctx, rc_h, &ctx->lists[0])) return rc;
  {
    GList& H = ctx->lists[0];
    const int64_t want = H.npairs + H.npairs * 3 / 10 + 4096;
    if (H.cap < want) {
      if (dev_alloc(ctx, &H.j, want) || dev_alloc(ctx, &H.mask, want)) return ORAC_ERR_CUDA;
      H.cap = want;
      for (int q = 1; q < 3; q++) {
        GList& L = ctx->lists[q];
        if (dev_alloc(ctx, &L.j, want) || dev_alloc(ctx, &L.mask, want)) return ORAC_ERR_CUDA;
        L.cap = want;
      }
      if (int rc = list_build_cells(ctx, rc_h, &ctx->lists[0])) return rc;
    }
  }
  {
    ShellRadii r1 = r;
    r1.rcuth = r.rcutl;
    r1.rtolh = 0.0;
    if (int rc = md_phony(ctx, r1, 'h')) return rc;
    ShellRadii r2 = r1;
    r2.rcutl = r.rcutm;
    r2.rtoll = 0.0;
    if (int rc = md_phony(ctx, r2, 'l')) return rc;
  }
  if (ctx->variant == VAR_ALCH) ctx->nlistqq = -1;  // built with this setup's constraints
  if (ctx->ne.on && ctx->variant == VAR_ALCH) {
    // the schedule's starting lambdas before the first forces
    const double tn0 = S.dth / ((double)S.lrespa * S.mrespa * S.n1respa * S.n0respa);
    if (int rc = ne_init(ctx, tn0)) return rc;
  }
  if (int rc = md_forces_shell(ctx, S, 'm', LM, true, S.e, true)) return rc;
  if (int rc = md_alch_m(ctx, S, false)) return rc;  // (systems without N1 pairs; else with the N1 level below)
  if (int rc = md_forces_shell(ctx, S, 'l', LL, true, S.e + 8, true)) return rc;
  if (int rc = md_forces_shell(ctx, S, 'h', LH, true, S.e + 16, true)) return rc;
  for (int l = LN1; l <= LN0; l++) {
    if (!S.ffix[l]) continue;
    CK(cudaMemsetAsync(S.ffix[l], 0, sizeof(unsigned long long) * 3 * (size_t)N, ctx->stream));
    if (int rc = md_forces_intra(ctx, S, l, false)) return rc;
  }
  {
    ShellRadii rr = ctx->sh;
    rr.rcutl = rr.rcutm;
    if (int rc = md_phony(ctx, rr, 'l')) return rc;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  S.ready = true;
  return ORAC_OK;
}

// Run nsteps outer steps.  Every `energy_every` steps (0: never) one record
// of ORAC_MD_REC = 16 doubles is written to rec (host): step, ekin, U_M (LJ,
// Coul), U_L (LJ, Coul), U_H (LJ, Coul), E_rec, econst, total, flag,
// bonded (bonds, bends, torsions, impropers), 1-4 + intra-group, erf
// corrections, 0.
int orac_gpu_md_set_thermostat(orac_gpu_ctx* ctx, double temp, double nu_com, double nu_solute,
                               double nu_solvent) {
  ParamGenBump bump(ctx);  // the step graphs gain the thermostat passes
  if (!ctx) return ORAC_ERR_PARAM;
  if (md_nupdte(ctx) > 0) return ctx_fail(ctx, ORAC_ERR_STATE, "set the thermostats before orac_gpu_md_setup");
  if (temp <= 0.0) {
    ctx->thermo.on = false;
    bump.arm();
    return ORAC_OK;
  }
  const double nu[3] = {nu_com, nu_solute, nu_solvent};
  for (double x : nu)
    if (!(x > 0.0 && std::isfinite(x))) return ctx_fail(ctx, ORAC_ERR_PARAM, "thermostat frequency %g cm^-1", x);
  if (!std::isfinite(temp)) return ctx_fail(ctx, ORAC_ERR_PARAM, "temperature");
  bump.arm();
  ctx->thermo.on = true;
  ctx->thermo.temp = temp;
  for (int k = 0; k < 3; k++) ctx->thermo.nu[k] = nu[k];
  return ORAC_OK;
}

int orac_gpu_md_set_thermostat_state(orac_gpu_ctx* ctx, const double* eta, const double* etap) {
  if (!ctx || !eta || !etap) return ORAC_ERR_PARAM;
  MdState* S = ctx->md;
  if (!S || !S->ready || !S->th) return ctx_fail(ctx, ORAC_ERR_STATE, "no thermostats (md_set_thermostat, md_setup)");
  for (int k = 0; k < 3; k++)
    if (!std::isfinite(eta[k]) || !std::isfinite(etap[k])) return ctx_fail(ctx, ORAC_ERR_PARAM, "thermostat state");
  CK(cudaSetDevice(ctx->device));
  ThermoDev T;
  CK(cudaMemcpyAsync(&T, S->th, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < 3; k++) {
    T.eta[k] = eta[k];
    T.etap[k] = etap[k];
    T.s[k] = std::exp(-T.tm4 * etap[k]);
  }
  CK(cudaMemcpyAsync(S->th, &T, sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return ORAC_OK;
}

int orac_gpu_md_thermostat(orac_gpu_ctx* ctx, double* out) {
  if (!ctx || !out) return ORAC_ERR_PARAM;
  MdState* S = ctx->md;
  if (!S || !S->ready || !S->th) return ctx_fail(ctx, ORAC_ERR_STATE, "no thermostats (md_set_thermostat, md_setup)");
  CK(cudaSetDevice(ctx->device));
  ThermoDev T;
  CK(cudaMemcpyAsync(&T, S->th, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double e = 0.0;
  for (int k = 0; k < 3; k++) {
    out[k] = T.eta[k];
    out[3 + k] = T.etap[k];
    out[6 + k] = T.q[k];
    out[9 + k] = S->th_ndf[k];
    e += T.ndfkt[k] * T.eta[k] + 0.5 * T.q[k] * T.etap[k] * T.etap[k];
  }
  out[12] = e;
  return ORAC_OK;
}

int orac_gpu_md_run(orac_gpu_ctx* ctx, int nsteps, int energy_every, double* rec) {
  return md_run_impl(ctx, nsteps, energy_every, rec, false);
}

// Queue nsteps steps without waiting (no energies, no status check); pair
// with orac_gpu_md_collect.
int orac_gpu_md_run_async(orac_gpu_ctx* ctx, int nsteps) { return md_run_impl(ctx, nsteps, 0, nullptr, true); }

// Wait for queued steps, collect the profiling events of the last step and
// check the run's status flags.
int orac_gpu_md_collect(orac_gpu_ctx* ctx) {
  if (!ctx) return ORAC_ERR_PARAM;
  MdState& S = *md_of(ctx);
  if (!S.h_flag) return ctx_fail(ctx, ORAC_ERR_STATE, "md_setup not called");
  if (S.flag_step != S.step) {
    // steps were queued since the last read-back (md_get_state reads the
    // flags with the state): wait for them and read the flags
    CK(cudaMemcpyAsync(S.h_flag, S.flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    S.flag_step = S.step;
  }
  if (ctx->prof && S.last_kind >= 0)
    if (int rc = prof_collect(ctx, S.pslot[S.last_kind][0], S.pslot[S.last_kind][1])) return rc;
  S.last_kind = -1;
  const int flag = *S.h_flag;
  if (flag & 1) return ctx_fail(ctx, ORAC_ERR_CAPACITY, "SHAKE/RATTLE did not converge");
  if (flag & 2) return ctx_fail(ctx, ORAC_ERR_CAPACITY, "neighbour list capacity exceeded during the run");
  return ORAC_OK;
}

int orac_gpu_md_get_state(orac_gpu_ctx* ctx, double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  if (!ctx) return ORAC_ERR_PARAM;
  MdState& S = *md_of(ctx);
  if (!S.ready) return ctx_fail(ctx, ORAC_ERR_STATE, "md_setup not called");
  double* dst[6] = {x, y, z, vx, vy, vz};
  const double* src[6] = {S.x, S.x + ctx->N, S.x + 2 * (size_t)ctx->N, S.v, S.v + ctx->N, S.v + 2 * (size_t)ctx->N};
  if (int rc = copy_runs(ctx, dst, src, cudaMemcpyDeviceToHost)) return rc;
  // the status flags travel with the state: a following md_collect need not
  // wait again
  CK(cudaMemcpyAsync(S.h_flag, S.flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  S.flag_step = S.step;
  return ORAC_OK;
}

int orac_gpu_md_set_state(orac_gpu_ctx* ctx, const double* x, const double* y, const double* z, const double* vx,
                          const double* vy, const double* vz) {
  if (!ctx) return ORAC_ERR_PARAM;
  MdState& S = *md_of(ctx);
  if (!S.ready) return ctx_fail(ctx, ORAC_ERR_STATE, "md_setup not called");
  const double* src[6] = {x, y, z, vx, vy, vz};
  double* dst[6] = {S.x, S.x + ctx->N, S.x + 2 * (size_t)ctx->N, S.v, S.v + ctx->N, S.v + 2 * (size_t)ctx->N};
  return copy_runs(ctx, dst, src, cudaMemcpyHostToDevice);
}

int orac_gpu_md_records(orac_gpu_ctx* ctx, int max, double* out, int64_t* n_total, int reset) {
  if (!ctx || max < 0 || (max > 0 && !out)) return ORAC_ERR_PARAM;
  MdState& S = *md_of(ctx);
  if (!S.ready) return ctx_fail(ctx, ORAC_ERR_STATE, "md_setup not called");
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  unsigned long long n = 0;
  CK(cudaMemcpy(&n, S.rec_n, sizeof(n), cudaMemcpyDeviceToHost));
  if (n_total) *n_total = (int64_t)n;
  const unsigned long long kept = n < (unsigned long long)S.rec_cap ? n : (unsigned long long)S.rec_cap;
  const unsigned long long take = kept < (unsigned long long)max ? kept : (unsigned long long)max;
  for (unsigned long long k = 0; k < take; k++) {  // oldest of the newest `take` first
    const unsigned long long idx = (n - take + k) % (unsigned long long)S.rec_cap;
    CK(cudaMemcpy(out + ORAC_MD_REC * k, S.rec + ORAC_MD_REC * idx, sizeof(double) * ORAC_MD_REC,
                  cudaMemcpyDeviceToHost));
  }
  if (reset) CK(cudaMemset(S.rec_n, 0, sizeof(unsigned long long)));
  return ORAC_OK;
}

int orac_gpu_md_set_graphs(orac_gpu_ctx* ctx, int on) {
  if (!ctx) return ORAC_ERR_PARAM;
  md_of(ctx)->use_graph = on != 0;
  return ORAC_OK;
}

}  // extern "C"

// capture (once) the step graph of one kind: 0 plain step, 1 step with list update
static int md_capture(orac_gpu_ctx* ctx, MdState& S, int kind) {
  bool any = false;
  for (int k = 0; k < 4; k++) any = any || S.gexec[k];
  if (any && (S.graphs_shared != ctx->shared_device || S.graphs_gen != ctx->param_gen)) {
    // captured for the other device-sharing mode, or before a parameter
    // changed (a new lambda, REM factor, box, ...): capture again
    for (int k = 0; k < 4; k++) {
      if (S.gexec[k]) cudaGraphExecDestroy(S.gexec[k]);
      if (S.graph[k]) cudaGraphDestroy(S.graph[k]);
      S.gexec[k] = nullptr;
      S.graph[k] = nullptr;
    }
  }
  S.graphs_shared = ctx->shared_device;
  S.graphs_gen = ctx->param_gen;
  if (S.gexec[kind]) return ORAC_OK;
  // listqq is built with synchronous copies: never inside the capture
  if (md_alch_intra(ctx) && ctx->nlistqq < 0)
    if (int rc = alch_listqq_build(ctx)) return rc;
  const int64_t l0 = ctx->launches;
  S.pslot[kind][0] = ctx->prof_next;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = md_step(ctx, S, (kind & 1) != 0, (kind & 2) != 0);
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  CK(ce);
  S.graph[kind] = g;
  CK(cudaGraphInstantiate(&S.gexec[kind], g, 0));
  S.pslot[kind][1] = ctx->prof_next;
  S.kpg[kind] = ctx->launches - l0;
  ctx->launches = l0;
  return ORAC_OK;
}

// ---- hooks of the batch driver (batch.cu)
int md_step_graph(orac_gpu_ctx* ctx, int kind, cudaGraph_t* out) {
  MdState& S = *md_of(ctx);
  if (!S.ready) return ctx_fail(ctx, ORAC_ERR_STATE, "md_setup not called");
  if (kind < 0 || kind > 3) return ctx_fail(ctx, ORAC_ERR_PARAM, "step graph kind %d", kind);
  if (int rc = md_capture(ctx, S, kind)) return rc;
  *out = S.graph[kind];
  return ORAC_OK;
}

int md_advance(orac_gpu_ctx* ctx, int nsteps, int kind) {
  MdState& S = *md_of(ctx);
  S.step += nsteps;
  ctx->launches += S.kpg[kind & 3] * nsteps;
  return ORAC_OK;
}

long long md_step_index(orac_gpu_ctx* ctx) { return ctx->md ? ctx->md->step : -1; }
int md_nupdte(orac_gpu_ctx* ctx) { return ctx->md && ctx->md->ready ? ctx->md->nupdte : -1; }

int md_check_flags(orac_gpu_ctx* ctx) {
  MdState& S = *md_of(ctx);
  int flag = 0;
  CK(cudaMemcpy(&flag, S.flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag & 1) return ctx_fail(ctx, ORAC_ERR_CAPACITY, "SHAKE/RATTLE did not converge");
  if (flag & 2) return ctx_fail(ctx, ORAC_ERR_CAPACITY, "neighbour list capacity exceeded during the run");
  return ORAC_OK;
}

static int md_run_impl(orac_gpu_ctx* ctx, int nsteps, int energy_every, double* rec, bool async) {
  if (!ctx) return ORAC_ERR_PARAM;
  MdState& S = *md_of(ctx);
  if (!S.ready) return ctx_fail(ctx, ORAC_ERR_STATE, "md_setup not called");
  CK(cudaSetDevice(ctx->device));
  int nrec = 0;
  for (int k = 0; k < nsteps; k++) {
    const bool update = (S.step % S.nupdte) == 0 && S.step > 0;
    const bool energy = energy_every > 0 && ((k + 1) % energy_every == 0);
    if (S.use_graph && !energy) {
      const int kind = update ? 1 : 0;
      // both kinds at once: the first list-update step of a run then pays
      // for no capture
      if (int rc = md_capture(ctx, S, kind)) return rc;
      if (int rc = md_capture(ctx, S, kind ^ 1)) return rc;
      CK(cudaGraphLaunch(S.gexec[kind], ctx->stream));
      ctx->launches += S.kpg[kind];
      S.last_kind = kind;
      if (ctx->prof && !async) {
        CK(cudaStreamSynchronize(ctx->stream));
        if (int rc = prof_collect(ctx, S.pslot[kind][0], S.pslot[kind][1])) return rc;
      }
    } else {
      const int p0 = ctx->prof_next;
      if (int rc = md_step(ctx, S, update, energy)) return rc;
      if (ctx->prof) {
        CK(cudaStreamSynchronize(ctx->stream));
        if (int rc = prof_collect(ctx, p0, ctx->prof_next)) return rc;
        ctx->prof_next = p0;
      }
    }
    S.step++;
    if (energy) {
      double e[96];
      int flag = 0;
      CK(cudaMemcpyAsync(e, S.e, sizeof(double) * 96, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(&flag, S.flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      double* r = rec + ORAC_MD_REC * (size_t)nrec++;
      r[0] = (double)S.step;
      r[1] = e[40];
      r[2] = e[4] + e[0] + e[6];  // M: ucnp + ucns + ucnsp
      r[3] = e[5] + e[1] + e[7];  // M: ucop + ucos + ucosp
      r[4] = e[12] + e[8] + e[14];
      r[5] = e[13] + e[9] + e[15];
      r[6] = e[20] + e[16] + e[22];
      r[7] = e[21] + e[17] + e[23];
      r[8] = 0.5 * e[24];
      r[9] = S.econst;
      r[12] = r[13] = r[14] = r[15] = 0.0;
      for (int q = E_BOND; q < E_14; q++) r[12] += e[q];
      for (int q = E_14; q < E_ERF; q++) r[13] += e[q];
      for (int q = E_ERF; q < E_DUDL; q++) r[14] += e[q];
      r[14] += e[E_AQQ] + e[E_AQQ + 1];
      // dU/dlambda of the alchemical windows: shells, PME, erf corrections,
      // fnb14_alchemy, ferrf_alchemy_add, self term
      if (ctx->variant == VAR_REM)  // REM: the shells' segment energy (rem_pot(3))
        for (int q = E_DUDL; q < E_DUDL + 3; q++) r[15] += e[q];
      if (ctx->variant == VAR_ALCH && ctx->d_dq) {
        for (int q = E_DUDL; q < E_DUDL + 7; q++) r[15] += e[q];
        r[15] += ctx->self_dudl;
      }
      if (md_ne(ctx)) {  // a non-equilibrium schedule: the work so far (wrk_alchemy)
        CK(cudaMemcpy(&r[15], &ctx->d_ne->wrk, sizeof(double), cudaMemcpyDeviceToHost));
      }
      r[10] = r[1] + r[2] + r[3] + r[4] + r[5] + r[6] + r[7] + r[8] + r[9] + r[12] + r[13] + r[14];
      if (S.th) {  // the thermostats' energy, in the total (the extended system's)
        ThermoDev T;
        CK(cudaMemcpy(&T, S.th, sizeof(T), cudaMemcpyDeviceToHost));
        double et = 0.0;
        for (int q = 0; q < 3; q++) et += T.ndfkt[q] * T.eta[q] + 0.5 * T.q[q] * T.etap[q] * T.etap[q];
        r[10] += et;
        // in column 15 where it has no other use (no alchemy, REM or schedule)
        if (ctx->variant != VAR_REM && !(ctx->variant == VAR_ALCH && ctx->d_dq) && !md_ne(ctx)) r[15] = et;
      }
      r[11] = (double)flag;
    }
  }
  if (async) return ORAC_OK;
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, S.flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (flag & 1) return ctx_fail(ctx, ORAC_ERR_CAPACITY, "SHAKE/RATTLE did not converge");
  if (flag & 2) return ctx_fail(ctx, ORAC_ERR_CAPACITY, "neighbour list capacity exceeded during the run");
  return ORAC_OK;
}
