// Bonded intramolecular forces of mts_intra_n0 / mts_intra_n1: harmonic
// stretching (fpbond, src/fpbond.f), bending with Urey-Bradley and
// stretch-stretch coupling (fpbend, src/fpbend.f), proper torsions as
// Chebyshev polynomials of cos(phi) (fptors, src/fptors.f) and improper
// torsions (fitors, src/fitors.f).  One thread per term, FP64 geometry,
// forces added with FP64 atomics (host entry points) or into a 64-bit
// fixed-point level accumulator (the MD driver), so the sum does not depend
// on the order of the atomics.
//
// A torsion whose atoms are collinear (|sin1 sin2 sin3| < 1e-25) is skipped;
// ORAC instead jitters the atoms with its random generator and retries
// (src/fptors.f:98-130).  Multiplicities other than 1..8 are not evaluated
// (ORAC's special forms 12 and 14 are not used by these systems).
#include <cmath>

#include "common.cuh"

namespace {

struct BondedArgs {
  int N;
  const double* x;  // [3N] Cartesian x|y|z
  const int* ss;    // ss_index per atom (1 solute, 2 solvent)
  int mask;         // BK_* kinds evaluated
  int nb, nbend, nt, nit;
  const int2* bij;
  const double2* bpar;
  const int4* aijk;
  const double* apot;
  const int4* tijkl;
  const double2* tpar;
  const int4* iijkl;
  const double4* ipar;
  double* f;                  // [3N] FP64 output, or
  unsigned long long* ffix;   // [3N] fixed-point output
  unsigned long long* ffix_t; // [3N] fixed-point output of the proper torsions (their own r-RESPA level)
  double* e;                  // [8] (bond, bend, tors, itors) x (slt, slv), or null
};

template <bool TORS = false>
__device__ __forceinline__ void put(const BondedArgs& A, int a, double fx, double fy, double fz) {
  unsigned long long* ff = TORS ? A.ffix_t : A.ffix;
  if (ff) {
    long long q = __double2ll_rn(fx * ORAC_FSCALE);
    if (q) atomicAdd(ff + a, (unsigned long long)q);
    q = __double2ll_rn(fy * ORAC_FSCALE);
    if (q) atomicAdd(ff + A.N + a, (unsigned long long)q);
    q = __double2ll_rn(fz * ORAC_FSCALE);
    if (q) atomicAdd(ff + 2 * A.N + a, (unsigned long long)q);
  } else {
    atomicAdd(A.f + a, fx);
    atomicAdd(A.f + A.N + a, fy);
    atomicAdd(A.f + 2 * A.N + a, fz);
  }
}

__device__ __forceinline__ void pos(const BondedArgs& A, int a, double* r) {
  r[0] = A.x[a];
  r[1] = A.x[A.N + a];
  r[2] = A.x[2 * A.N + a];
}

__device__ bool cheb(int n, double c, double* t, double* dt) {
  const double c2 = c * c;
  switch (n) {
    case 1: *t = c; *dt = 1.0; return true;
    case 2: *t = 2.0 * c2 - 1.0; *dt = 4.0 * c; return true;
    case 3: *t = 4.0 * c2 * c - 3.0 * c; *dt = 12.0 * c2 - 3.0; return true;
    case 4: *t = 8.0 * c2 * c2 - 8.0 * c2 + 1.0; *dt = 32.0 * c2 * c - 16.0 * c; return true;
    case 5:
      *t = 16.0 * c2 * c2 * c - 20.0 * c2 * c + 5.0 * c;
      *dt = 80.0 * c2 * c2 - 60.0 * c2 + 5.0;
      return true;
    case 6:
      *t = 32.0 * c2 * c2 * c2 - 48.0 * c2 * c2 + 18.0 * c2 - 1.0;
      *dt = 192.0 * c2 * c2 * c - 192.0 * c2 * c + 36.0 * c;
      return true;
    case 7:
      *t = 64.0 * c2 * c2 * c2 * c - 112.0 * c2 * c2 * c + 56.0 * c2 * c - 7.0 * c;
      *dt = 448.0 * c2 * c2 * c2 - 560.0 * c2 * c2 + 168.0 * c2 - 7.0;
      return true;
    case 8:
      *t = 128.0 * c2 * c2 * c2 * c2 - 256.0 * c2 * c2 * c2 + 160.0 * c2 * c2 - 32.0 * c2 + 1.0;
      *dt = 1024.0 * c2 * c2 * c2 * c - 1536.0 * c2 * c2 * c + 640.0 * c2 * c - 64.0 * c;
      return true;
    default: return false;
  }
}

// cos(phi) of the dihedral 1-2-3-4 and its gradient (src/fptors.f:69-176);
// sgn carries the orientation (r21 x r32) . r43.  absq selects fptors'
// |1 - cos^2| under the square roots (fitors has none).
__device__ bool torsion_geom(const BondedArgs& A, int4 l, bool absq, double* coa, double g[4][3], double* sgn) {
  double r1[3], r2[3], r3[3], r4[3];
  pos(A, l.x, r1);
  pos(A, l.y, r2);
  pos(A, l.z, r3);
  pos(A, l.w, r4);
  double d21[3], d32[3], d43[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    d21[k] = r2[k] - r1[k];
    d32[k] = r3[k] - r2[k];
    d43[k] = r4[k] - r3[k];
  }
  const double rsq21 = d21[0] * d21[0] + d21[1] * d21[1] + d21[2] * d21[2];
  const double rsq32 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
  const double rsq43 = d43[0] * d43[0] + d43[1] * d43[1] + d43[2] * d43[2];
  // every quotient of the reference's expressions as a product of
  // reciprocal square roots: 1/|r| for the three bonds and 1/sin for the
  // three angles (a zero or negative 1 - cos^2 gives inf or NaN, which the
  // degeneracy test below rejects as it rejects a zero sine)
  const double ir21 = rsqrt(rsq21), ir32 = rsqrt(rsq32), ir43 = rsqrt(rsq43);
  const double cb1 = (d21[0] * d32[0] + d21[1] * d32[1] + d21[2] * d32[2]) * (ir21 * ir32);
  const double cb2 = (d43[0] * d32[0] + d43[1] * d32[1] + d43[2] * d32[2]) * (ir43 * ir32);
  const double cb3 = (d21[0] * d43[0] + d21[1] * d43[1] + d21[2] * d43[2]) * (ir21 * ir43);
  const double q1 = absq ? fabs(1.0 - cb1 * cb1) : 1.0 - cb1 * cb1;
  const double q2 = absq ? fabs(1.0 - cb2 * cb2) : 1.0 - cb2 * cb2;
  const double q3 = absq ? fabs(1.0 - cb3 * cb3) : 1.0 - cb3 * cb3;
  const double is1 = rsqrt(q1), is2 = rsqrt(q2), is3 = rsqrt(q3);
  const double sb1 = q1 * is1, sb2 = q2 * is2, sb3 = q3 * is3;
  const double aux = sb1 * sb2;
  if (!(fabs(aux * sb3) >= 1e-25)) return false;
  const double iaux = is1 * is2;
  double c = (cb1 * cb2 - cb3) * iaux;
  if (c > 1.0 && c < 1.000001) c = 1.0;
  if (c < -1.0 && c > -1.000001) c = -1.0;
  const double aux1 = cb1 * sb2, aux2 = sb1 * cb2;
  const double auxa = -(aux1 * c + aux2) * iaux;
  const double auxb = -(aux2 * c + aux1) * iaux;
  const double auxc = sb3 * iaux;
  const double ia1 = ir21 * ir32 * is1, ia2 = ir32 * ir43 * is2, ia3 = ir21 * ir43 * is3;
  const double c1a = cb1 * ir21 * ir21 * is1, c1b = cb1 * ir32 * ir32 * is1;
  const double c2a = cb2 * ir32 * ir32 * is2, c2b = cb2 * ir43 * ir43 * is2;
  const double c3a = cb3 * ir21 * ir21 * is3, c3b = cb3 * ir43 * ir43 * is3;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double v21 = d21[k], v32 = d32[k], v43 = d43[k];
    const double b11 = v32 * ia1 - c1a * v21;
    const double b13 = -v21 * ia1 + c1b * v32;
    const double b12 = -b13 - b11;
    const double b22 = v43 * ia2 - c2a * v32;
    const double b24 = -v32 * ia2 + c2b * v43;
    const double b23 = -b22 - b24;
    const double b31 = v43 * ia3 - c3a * v21;
    const double b33 = v21 * ia3 - c3b * v43;
    g[0][k] = auxa * b11 + auxc * b31;
    g[1][k] = auxa * b12 + auxb * b22 - auxc * b31;
    g[2][k] = auxa * b13 + auxb * b23 + auxc * b33;
    g[3][k] = auxb * b24 - auxc * b33;
  }
  *coa = c;
  const double xn = d21[1] * d32[2] - d32[1] * d21[2];
  const double yn = d21[2] * d32[0] - d32[2] * d21[0];
  const double zn = d21[0] * d32[1] - d32[0] * d21[1];
  *sgn = xn * d43[0] + yn * d43[1] + zn * d43[2];
  return true;
}

__device__ __forceinline__ double warp_sumd(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// e[B + type] += v with a constant index (type 0 solute, 1 solvent): the
// energy array stays in registers
template <int B>
__device__ __forceinline__ void eadd(double* e, int type, double v) {
  if (type == 0)
    e[B] += v;
  else
    e[B + 1] += v;
}

__global__ void k_bonded(const BondedArgs A) {
  pdl_enter();
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if ((A.mask & BK_BOND) && t < A.nb) {
    // fpbond (src/fpbond.f:44-75)
    const int2 l = A.bij[t];
    const double2 p = A.bpar[t];  // (r0, k)
    double ra[3], rb[3];
    pos(A, l.x, ra);
    pos(A, l.y, rb);
    const double x21 = rb[0] - ra[0], y21 = rb[1] - ra[1], z21 = rb[2] - ra[2];
    // correctly rounded: near its minimum (r - r0)^2 cancels to a few ulp of r
    const double rs21 = sqrt(x21 * x21 + y21 * y21 + z21 * z21);
    const double qforce = -2.0 * p.y * (p.x - rs21) / rs21;
    put(A, l.x, qforce * x21, qforce * y21, qforce * z21);
    put(A, l.y, -qforce * x21, -qforce * y21, -qforce * z21);
    eadd<0>(e, A.ss[l.x] - 1, p.y * (rs21 - p.x) * (rs21 - p.x));
  }
  t -= A.nb;
  if ((A.mask & BK_BEND) && t >= 0 && t < A.nbend) {
    // fpbend (src/fpbend.f:60-180)
    const int4 l = A.aijk[t];
    const double* P = A.apot + 7 * t;
    const double pota = P[0], potb = P[1], potc = P[2], potd = P[3], pote = P[4], potf = P[5], potg = P[6];
    if (fabs(potb) >= 1e-12) {
      const double pi = 3.14159265358979323846;
      double r1[3], r2[3], r3[3];
      pos(A, l.x, r1);
      pos(A, l.y, r2);
      pos(A, l.z, r3);
      const double d12[3] = {r1[0] - r2[0], r1[1] - r2[1], r1[2] - r2[2]};
      const double d32[3] = {r3[0] - r2[0], r3[1] - r2[1], r3[2] - r2[2]};
      const double rs12 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
      const double rs32 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
      const double ir12 = rsqrt(rs12), ir32 = rsqrt(rs32), idcc2 = ir12 * ir32;
      const double irs12 = ir12 * ir12, irs32 = ir32 * ir32;
      double cb = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) * idcc2;
      if (fabs(cb) > 1.0) cb = cb > 0 ? 1.0 : -1.0;
      const double sb = sqrt(1.0 - cb * cb);
      const double bb = acos(cb);
      const bool linear = fabs(pota - pi) < 0.01;
      const double qforce = (linear || sb < 1e-6) ? -2.0 * potb : 2.0 * potb * (bb - pota) / sb;
      double u1[3], u3[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        u1[k] = d32[k] * idcc2 - cb * d12[k] * irs12;
        u3[k] = d12[k] * idcc2 - cb * d32[k] * irs32;
      }
      put(A, l.x, qforce * u1[0], qforce * u1[1], qforce * u1[2]);
      put(A, l.z, qforce * u3[0], qforce * u3[1], qforce * u3[2]);
      put(A, l.y, -qforce * (u1[0] + u3[0]), -qforce * (u1[1] + u3[1]), -qforce * (u1[2] + u3[2]));
      const int ty = A.ss[l.x] - 1;
      eadd<2>(e, ty, linear ? 2.0 * potb * (cb + 1.0) : potb * (bb - pota) * (bb - pota));
      if (fabs(potd) > 1e-5 && (fabs(pote) < 1e-5 || fabs(potf) > 1e-5)) {
        // Urey-Bradley 1-3 spring
        const double d31[3] = {r3[0] - r1[0], r3[1] - r1[1], r3[2] - r1[2]};
        const double rsp31 = sqrt(d31[0] * d31[0] + d31[1] * d31[1] + d31[2] * d31[2]);
        const double q = -2.0 * potd * (potc - rsp31) / rsp31;
        put(A, l.x, q * d31[0], q * d31[1], q * d31[2]);
        put(A, l.z, -q * d31[0], -q * d31[1], -q * d31[2]);
        eadd<2>(e, ty, potd * (rsp31 - potc) * (rsp31 - potc));
      }
      bool coupling = false;
      double k12 = 0, rr1 = 0, rr2 = 0;
      if (fabs(potd) > 1e-5 && fabs(pote) > 1e-5 && fabs(potf) < 1e-5) {
        coupling = true;
        k12 = potd;
        rr1 = potc;
        rr2 = pote;
      }
      if (fabs(pote) > 1e-5 && fabs(potf) > 1e-5 && fabs(potg) > 1e-5) {
        coupling = true;
        k12 = pote;
        rr1 = potf;
        rr2 = potg;
      }
      if (coupling) {
        const double rsp12 = sqrt(rs12), rsp32 = sqrt(rs32);
        const double qf = k12 * (rsp12 - rr1), pf = k12 * (rsp32 - rr2);
        const double a1[3] = {d12[0] / rsp12, d12[1] / rsp12, d12[2] / rsp12};
        const double a2[3] = {d32[0] / rsp32, d32[1] / rsp32, d32[2] / rsp32};
        put(A, l.x, -pf * a1[0], -pf * a1[1], -pf * a1[2]);
        put(A, l.y, pf * a1[0] + qf * a2[0], pf * a1[1] + qf * a2[1], pf * a1[2] + qf * a2[2]);
        put(A, l.z, -qf * a2[0], -qf * a2[1], -qf * a2[2]);
        eadd<2>(e, ty, k12 * (rsp12 - rr1) * (rsp32 - rr2));
      }
    }
  }
  t -= A.nbend;
  if ((A.mask & BK_TORS) && t >= 0 && t < A.nt) {
    // fptors (src/fptors.f:178-263)
    const int4 l = A.tijkl[t];
    const double2 p = A.tpar[t];  // (+-n, V)
    const int tmp = (int)llround(p.x);
    const int n = tmp < 0 ? -tmp : tmp;
    const double sig = tmp < 0 ? -1.0 : 1.0;
    double coa, g[4][3], sgn, tt, dt;
    if (fabs(p.y) >= 1e-12 && n >= 1 && n <= 8 && torsion_geom(A, l, true, &coa, g, &sgn)) {
      cheb(n, coa, &tt, &dt);
      const double qforce = sig * dt * p.y;
      eadd<4>(e, A.ss[l.x] - 1, sig * (fabs(p.y) - tt * p.y));
      put<true>(A, l.x, qforce * g[0][0], qforce * g[0][1], qforce * g[0][2]);
      put<true>(A, l.y, qforce * g[1][0], qforce * g[1][1], qforce * g[1][2]);
      put<true>(A, l.z, qforce * g[2][0], qforce * g[2][1], qforce * g[2][2]);
      put<true>(A, l.w, qforce * g[3][0], qforce * g[3][1], qforce * g[3][2]);
    }
  }
  t -= A.nt;
  if ((A.mask & BK_ITORS) && t >= 0 && t < A.nit) {
    // fitors (src/fitors.f:74-262)
    const int4 l = A.iijkl[t];
    const double4 p = A.ipar[t];  // (pota, potb, potc)
    double coa, g[4][3], sgn;
    if (fabs(p.y) >= 1e-12 && torsion_geom(A, l, false, &coa, g, &sgn)) {
      double enrg = 0.0, qforce = 0.0;
      bool ok = true;
      if (p.z > 0.0) {
        double bb = acos(coa);
        const double aux4 = sgn >= 0 ? bb : -bb;
        if (aux4 < 0.0 && fabs(aux4) >= 1.57079) {
          bb = 2.0 * acos(-1.0) + aux4;
          if (fabs(p.x - bb) > 3.14159) bb = -2 * 3.14159 + bb;
        } else if (aux4 < 0.0 && fabs(aux4) < 1.57079) {
          bb = aux4;
          if (fabs(p.x - bb) > 3.14159) bb = 2 * 3.14159 + bb;
        } else {
          bb = aux4;
          if (fabs(p.x - bb) > 3.14159) bb = 2 * 3.14159 + bb;
          if (fabs(p.x - bb) > 3.14159) bb = -4 * 3.14159 + bb;
        }
        if (fabs(p.x) < 1e-3)
          qforce = 2.0 * p.y;
        else if (fabs(p.x - 3.14159) < 1e-3)
          qforce = -2.0 * p.y;
        else
          qforce = 2.0 * p.y * (bb - p.x) / sin(bb);
        enrg = p.y * (bb - p.x) * (bb - p.x);
      } else {
        const int tmp = (int)llround(p.x);
        const int n = tmp < 0 ? -tmp : tmp;
        const double sig = tmp < 0 ? -1.0 : 1.0;
        double tt, dt;
        ok = n >= 1 && n <= 8 && cheb(n, coa, &tt, &dt);
        if (ok) {
          enrg = sig * (fabs(p.y) - tt * p.y);
          qforce = sig * dt * p.y;
        }
      }
      if (ok) {
        eadd<6>(e, A.ss[l.x] - 1, enrg);
        put(A, l.x, qforce * g[0][0], qforce * g[0][1], qforce * g[0][2]);
        put(A, l.y, qforce * g[1][0], qforce * g[1][1], qforce * g[1][2]);
        put(A, l.z, qforce * g[2][0], qforce * g[2][1], qforce * g[2][2]);
        put(A, l.w, qforce * g[3][0], qforce * g[3][1], qforce * g[3][2]);
      }
    }
  }
  if (!A.e) return;
  __shared__ double s[8][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const double v = warp_sumd(e[q]);
    if (lane == 0) s[w][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double v = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) v += s[k][threadIdx.x];
    if (v != 0.0) atomicAdd(A.e + threadIdx.x, v);
  }
}

}  // namespace

int bonded_launch(orac_gpu_ctx* ctx, int mask, const double* d_x, double* d_f, unsigned long long* d_ffix,
                  double* d_e, unsigned long long* d_ffix_tors) {
  const BondedDev& B = ctx->bd;
  BondedArgs A;
  memset(&A, 0, sizeof(A));
  A.N = ctx->N;
  A.x = d_x;
  A.ss = B.ss;
  A.mask = mask;
  A.nb = B.nb;
  A.nbend = B.nbend;
  A.nt = B.nt;
  A.nit = B.nit;
  A.bij = B.bij;
  A.bpar = B.bpar;
  A.aijk = B.aijk;
  A.apot = B.apot;
  A.tijkl = B.tijkl;
  A.tpar = B.tpar;
  A.iijkl = B.iijkl;
  A.ipar = B.ipar;
  A.f = d_f;
  A.ffix = d_ffix;
  A.ffix_t = d_ffix_tors ? d_ffix_tors : d_ffix;
  A.e = d_e;
  const int n = B.nb + B.nbend + B.nt + B.nit;
  if (n == 0) return ORAC_OK;
  // 64 threads a block: the terms of one launch spread over four times the
  // SMs (each thread's FP64 chain sets the time, not the issue rate)
  orac_launch(k_bonded, (n + 63) / 64, 64, 0, ctx->stream, A);
  CKL();
  return ORAC_OK;
}
