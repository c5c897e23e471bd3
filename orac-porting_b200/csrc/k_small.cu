// List-driven correction kernels: fnb14 (src/fnb14.f:1-219), fnbgrp
// (src/fnbgrp.f:1-213) and ferrf (src/ferrf.f:1-244, erf_corr off).  One
// thread per listed pair.  These lists are short (hundreds to thousands of
// pairs) and their terms are large intramolecular values that cancel against
// the reciprocal sum, so they are evaluated in FP64; forces are accumulated
// with FP64 atomics.
#include <cmath>

#include "common.cuh"

namespace {

constexpr double AS_A1 = 0.2548296, AS_A2 = -0.28449674, AS_A3 = 1.4214137;
constexpr double AS_A4 = -1.453152, AS_A5 = 1.0614054, AS_QP = 0.3275911;

__device__ __forceinline__ double warp_sumd(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct SmallArgs {
  int kind;  // 0 fnb14, 1 fnbgrp, 2 ferrf, 3 fnb14_alchemy, 4 ferrf_alchemy_add
  int n;     // pairs
  int natom;
  const double* xyz;  // [3N] Cartesian
  const int* pairs;   // [2n] 1-based
  const int* ptype;   // fnb14: type14 (1-based into tab); fnbgrp: nbtype per atom
  const double* tab12;
  const double* tab6;
  const double* q;
  const int* ss;  // ss_index per atom
  double alpha, fudge, lj_fudge, twrtpi;
  int coul_mode;  // 1 Ewald erfc, 0 bare Coulomb
  int forces;
  double* f;  // [3N]
  double* e;  // [4]
  unsigned long long* ffix;  // [3N] fixed-point output instead of f (or null)
  // ferrf: d/dlambda of the correction for charges q(lambda) with dq/dlambda
  const double* dq;
  double* edq;
  // fnb14_alchemy, ferrf_alchemy_add: per atom (lambda LJ, lambda charge,
  // d(1-|lambda LJ|)/dlambda, d(1-|lambda charge|)/dlambda); the charges
  // q are the full ones; intramol skips same-species listqq pairs
  const double4* lam4;
  int intramol;
  // the work U(lambda) - U(lambda0) of fnb14_alchemy / ferrf_alchemy_add
  // (their dwrk) with the lambda0 of each atom in lam40, into *work
  const double4* lam40;
  double* work;
};

// Coupling factors of one pair of fnb14_alchemy (src/fnb14_alchemy.f:
// 149-177, 252-289) from the atoms' lambdas li, lj with the derivatives
// di, dj of their couplings 1-|l|: f scales the erfc (or LJ) term, f2 the
// erf term of the charges; df, df2 their derivatives.  An alchemical atom
// at lambda 0 counts as normal; one alchemical atom: its coupling; two of
// one lambda: full, with f2 = 1 - the product of couplings; two of
// different lambdas: none, f2 = - that product.
__device__ __forceinline__ void alch14_factors(double li, double lj, double di, double dj, bool charges, double* f,
                                               double* df, double* f2, double* df2) {
  const double ci = 1.0 - fabs(li), cj = 1.0 - fabs(lj);
  *f2 = 0.0;
  *df2 = 0.0;
  *df = 0.0;
  if (li == 0.0 && lj != 0.0) {
    *f = cj;
    *df = dj;
  } else if (li != 0.0 && lj == 0.0) {
    *f = ci;
    *df = di;
  } else if (li == 0.0 && lj == 0.0) {
    *f = 1.0;
  } else if (li != lj) {
    *f = 0.0;
    if (charges) {
      *f2 = -ci * cj;
      *df2 = -(di * cj + ci * dj);
    }
  } else {
    *f = 1.0;
    if (charges) {
      *f2 = 1.0 - ci * cj;
      *df2 = -(di * cj + ci * dj);
    }
  }
}

// e[B + type] += v with a constant index (type 0 solute, 1 solvent)
template <int B>
__device__ __forceinline__ void eadd(double* e, int type, double v) {
  if (type == 0)
    e[B] += v;
  else
    e[B + 1] += v;
}

__device__ __forceinline__ void small_body(const SmallArgs& A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double e[4] = {0, 0, 0, 0};
  double dedl = 0.0, wk = 0.0;
  if (t < A.n) {
    const int stride = A.kind == 4 ? 3 : 2;  // listqq carries facQ
    const int i1 = A.pairs[stride * t] - 1, i2 = A.pairs[stride * t + 1] - 1;
    const int type = A.ss[i1] - 1;
    const double xa = A.xyz[i1] - A.xyz[i2];
    const double ya = A.xyz[A.natom + i1] - A.xyz[A.natom + i2];
    const double za = A.xyz[2 * A.natom + i1] - A.xyz[2 * A.natom + i2];
    const double rsq = xa * xa + ya * ya + za * za;
    const double rsp = sqrt(rsq);
    const double rsqi = 1.0 / rsq;
    double qforce = 0.0;
    bool skip = false;
    if (A.kind == 4) {
      // ferrf_alchemy_add (src/ferrf_alchemy_add.f): the reciprocal sum of
      // the scaled charges gave the pair c_a c_b Q_a Q_b erf/r; subtract
      // (c_a c_b - facQ) of it, so one species keeps its full Coulomb
      // (facQ 1) and added and removed atoms do not see each other (0)
      const int facq = A.pairs[3 * t + 2];
      skip = A.intramol && facq != 0;
      if (!skip) {
        const double4 la = A.lam4[i1], lb = A.lam4[i2];
        const double ca = 1.0 - fabs(la.y), cb = 1.0 - fabs(lb.y);
        const double qab = A.q[i1] * A.q[i2];
        const double furpar = (ca * cb - (double)facq) * qab;
        const double alphar = A.alpha * rsp;
        const double qt = 1.0 / (1.0 + AS_QP * alphar);
        const double expcst = exp(-alphar * alphar);
        const double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
        const double erfst = 1.0 - erfcst;
        eadd<0>(e, type, -(furpar * erfst / rsp));
        qforce = -furpar * (erfst - A.twrtpi * alphar * expcst) / (rsp * rsq);
        dedl = -(la.w * cb + ca * lb.w) * qab * erfst / rsp;
        if (A.work) {
          const double4 la0 = A.lam40[i1], lb0 = A.lam40[i2];
          const double furpar0 = ((1.0 - fabs(la0.y)) * (1.0 - fabs(lb0.y)) - (double)facq) * qab;
          wk = -furpar * erfst / rsp + furpar0 * erfst / rsp;
        }
      }
    } else if (A.kind == 3) {
      // fnb14_alchemy, Ewald branch (src/fnb14_alchemy.f:225-341); ORAC
      // scales only the repulsive term of the LJ force by alch_fact (its
      // energy by alch_fact whole), restated as written
      const double4 la = A.lam4[i1], lb = A.lam4[i2];
      double af, daf, dum, ddum, aq, daq, aq2, daq2;
      alch14_factors(la.x, lb.x, la.z, lb.z, false, &af, &daf, &dum, &ddum);
      alch14_factors(la.y, lb.y, la.w, lb.w, true, &aq, &daq, &aq2, &daq2);
      const int lij = A.ptype[t] - 1;
      const double rspqi = rsqi / rsp;
      const double r6 = rsqi * rsqi * rsqi;
      const double r12 = r6 * r6;
      const double ssvir = af * 12.0 * A.tab12[lij] * r12 - 6.0 * A.tab6[lij] * r6;
      qforce = A.lj_fudge * ssvir * rsqi;
      const double elj = A.lj_fudge * (A.tab12[lij] * r12 - A.tab6[lij] * r6);
      eadd<0>(e, type, af * elj);
      const double alphar = A.alpha * rsp;
      const double qt = 1.0 / (1.0 + AS_QP * alphar);
      const double expcst = exp(-alphar * alphar);
      const double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
      const double erff = 1.0 - erfcst;
      const double qq = A.fudge * A.q[i1] * A.q[i2];
      eadd<2>(e, type, qq * (aq * erfcst + aq2 * erff) / rsp);
      qforce += qq * (aq * (erfcst + A.twrtpi * alphar * expcst) + aq2 * (erff - A.twrtpi * alphar * expcst)) * rspqi;
      dedl = daf * elj + qq * (daq * erfcst + daq2 * erff) / rsp;
      if (A.work) {
        const double4 la0 = A.lam40[i1], lb0 = A.lam40[i2];
        double af0, aq0, aq20;
        alch14_factors(la0.x, lb0.x, 0.0, 0.0, false, &af0, &dum, &ddum, &ddum);
        alch14_factors(la0.y, lb0.y, 0.0, 0.0, true, &aq0, &dum, &aq20, &ddum);
        wk = (af * elj + qq * (aq * erfcst + aq2 * erff) / rsp) - (af0 * elj + qq * (aq0 * erfcst + aq20 * erff) / rsp);
      }
    } else if (A.kind == 2) {
      // ferrf: subtract fudge q q erf(alpha r)/r
      const double furpar = (A.forces ? A.fudge : 1.0) * A.q[i1] * A.q[i2];
      const double alphar = A.alpha * rsp;
      const double qt = 1.0 / (1.0 + AS_QP * alphar);
      const double expcst = exp(-alphar * alphar);
      const double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
      const double erfst = 1.0 - erfcst;
      eadd<0>(e, type, -(furpar * erfst / rsp));
      qforce = -furpar * (erfst - A.twrtpi * alphar * expcst) / (rsp * rsq);
      if (A.dq)
        dedl = -(A.forces ? A.fudge : 1.0) * (A.dq[i1] * A.q[i2] + A.q[i1] * A.dq[i2]) * erfst / rsp;
    } else {
      int lij;
      if (A.kind == 0) {
        lij = A.ptype[t] - 1;
      } else {
        const int ta = A.ptype[i1], tb = A.ptype[i2];
        const int lj = ta > tb ? ta : tb, li = ta > tb ? tb : ta;
        lij = lj * (lj - 1) / 2 + li - 1;
      }
      const double lf = A.kind == 0 ? A.lj_fudge : 1.0;
      const double qf = A.kind == 0 ? A.fudge : 1.0;
      const double r6 = rsqi * rsqi * rsqi;
      const double r12 = r6 * r6;
      const double ssvir = 12.0 * A.tab12[lij] * r12 - 6.0 * A.tab6[lij] * r6;
      qforce = lf * ssvir * rsqi;
      eadd<0>(e, type, lf * (A.tab12[lij] * r12 - A.tab6[lij] * r6));
      const double furpar = qf * A.q[i1] * A.q[i2];
      if (A.coul_mode) {
        const double rspqi = rsqi / rsp;
        const double alphar = A.alpha * rsp;
        const double qt = 1.0 / (1.0 + AS_QP * alphar);
        const double expcst = exp(-alphar * alphar);
        const double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
        eadd<2>(e, type, furpar * erfcst / rsp);
        qforce += furpar * (erfcst + A.twrtpi * alphar * expcst) * rspqi;
      } else {
        const double sv = furpar / rsp;
        eadd<2>(e, type, sv);
        qforce += sv * rsqi;
      }
    }
    if (skip) {
    } else if (A.forces && A.ffix) {
      const double fv[3] = {qforce * xa, qforce * ya, qforce * za};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const long long q = __double2ll_rn(fv[d] * ORAC_FSCALE);
        if (q) {
          atomicAdd(A.ffix + d * A.natom + i1, (unsigned long long)q);
          atomicAdd(A.ffix + d * A.natom + i2, (unsigned long long)(-q));
        }
      }
    } else if (A.forces && A.f) {
      atomicAdd(A.f + i1, qforce * xa);
      atomicAdd(A.f + A.natom + i1, qforce * ya);
      atomicAdd(A.f + 2 * A.natom + i1, qforce * za);
      atomicAdd(A.f + i2, -qforce * xa);
      atomicAdd(A.f + A.natom + i2, -qforce * ya);
      atomicAdd(A.f + 2 * A.natom + i2, -qforce * za);
    }
  }
  __shared__ double s[8][4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const double x = warp_sumd(e[q]);
    if (lane == 0) s[w][q] = x;
  }
  __syncthreads();
  if (A.e && threadIdx.x < 4) {
    double x = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) x += s[k][threadIdx.x];
    if (x != 0.0) atomicAdd(A.e + threadIdx.x, x);
  }
  if (A.edq) {
    const double x = warp_sumd(dedl);
    if (lane == 0 && x != 0.0) atomicAdd(A.edq, x);
  }
  if (A.work) {
    const double x = warp_sumd(wk);
    if (lane == 0 && x != 0.0) atomicAdd(A.work, x);
  }
}

__global__ void k_small(const SmallArgs A) {
  pdl_enter();
  small_body(A);
}

// up to four pair lists of one kind in one launch, blockIdx.y the list:
// a block never spans two lists, so each keeps its own energy slots
constexpr int MAX_SEGS = 4;
struct SmallSegs {
  SmallArgs s[MAX_SEGS];
};

__global__ void k_small_segs(const SmallSegs S) {
  pdl_enter();
  small_body(S.s[blockIdx.y]);
}

__global__ void k_self(int n, const double* q, const int* ss, double* e) {
  pdl_enter();
  __shared__ double s[8][2];
  double v[2] = {0, 0};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    v[ss[t] - 1] += q[t] * q[t];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = 0; k < 2; k++) {
    const double x = warp_sumd(v[k]);
    if (lane == 0) s[w][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double x = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) x += s[k][threadIdx.x];
    atomicAdd(e + threadIdx.x, x);
  }
}

}  // namespace

int small_launch(orac_gpu_ctx* ctx, int kind, const double* d_xyz, const int* d_pairs, const int* d_ptype, int npairs,
                 const double* d_t12, const double* d_t6, double fudge, double lj_fudge, int coul_mode, int forces,
                 double* d_f, double* d_e, const int* d_ss) {
  return small_launch_x(ctx, kind, d_xyz, d_pairs, d_ptype, npairs, d_t12, d_t6, fudge, lj_fudge, coul_mode, forces,
                        d_f, d_e, d_ss, nullptr, nullptr);
}

static SmallArgs small_args(orac_gpu_ctx* ctx, int kind, const double* d_xyz, const int* d_pairs,
                            const int* d_ptype, int npairs, const double* d_t12, const double* d_t6, double fudge,
                            double lj_fudge, int coul_mode, int forces, double* d_f, double* d_e, const int* d_ss,
                            const double* d_q, unsigned long long* d_ffix, const double* d_dq, double* d_edq) {
  SmallArgs A;
  memset(&A, 0, sizeof(A));
  A.kind = kind;
  A.n = npairs;
  A.natom = ctx->N;
  A.xyz = d_xyz;
  A.pairs = d_pairs;
  A.ptype = d_ptype;
  A.tab12 = d_t12;
  A.tab6 = d_t6;
  A.q = d_q ? d_q : ctx->d_aqd;
  A.ss = d_ss;
  A.ffix = d_ffix;
  A.dq = (kind == 2 && d_edq) ? d_dq : nullptr;
  A.edq = (A.dq || kind >= 3) ? d_edq : nullptr;
  A.lam4 = ctx->d_lam4;
  A.intramol = ctx->alch_intramol;
  A.alpha = ctx->alphal;
  A.fudge = fudge;
  A.lj_fudge = lj_fudge;
  A.twrtpi = 2.0 / std::sqrt(4.0 * std::atan(1.0));
  A.coul_mode = coul_mode;
  A.forces = forces;
  A.f = d_f;
  A.e = d_e;
  return A;
}

int small_launch_x(orac_gpu_ctx* ctx, int kind, const double* d_xyz, const int* d_pairs, const int* d_ptype,
                   int npairs, const double* d_t12, const double* d_t6, double fudge, double lj_fudge,
                   int coul_mode, int forces, double* d_f, double* d_e, const int* d_ss, const double* d_q,
                   unsigned long long* d_ffix, const double* d_dq, double* d_edq) {
  const SmallArgs A = small_args(ctx, kind, d_xyz, d_pairs, d_ptype, npairs, d_t12, d_t6, fudge, lj_fudge, coul_mode,
                                 forces, d_f, d_e, d_ss, d_q, d_ffix, d_dq, d_edq);
  if (npairs > 0) {
    orac_launch(k_small, (npairs + 255) / 256, 256, 0, ctx->stream, A);
    CKL();
  }
  return ORAC_OK;
}

int ferrf_launch_lists(orac_gpu_ctx* ctx, int nlist, const int* const* d_pairs, const int* npairs,
                       const double* fudge, const int* forces, double* const* d_e, const double* d_xyz,
                       const int* d_ss, const double* d_q, unsigned long long* d_ffix, const double* d_dq,
                       double* d_edq) {
  SmallSegs S;
  memset(&S, 0, sizeof(S));
  int ns = 0, nmax = 0;
  for (int k = 0; k < nlist && ns < MAX_SEGS; k++) {
    if (npairs[k] <= 0) continue;
    S.s[ns++] = small_args(ctx, 2, d_xyz, d_pairs[k], nullptr, npairs[k], nullptr, nullptr, fudge[k], 1.0, 1,
                           forces[k], nullptr, d_e[k], d_ss, d_q, d_ffix, d_dq, d_edq);
    nmax = npairs[k] > nmax ? npairs[k] : nmax;
  }
  if (ns == 0) return ORAC_OK;
  orac_launch(k_small_segs, dim3((nmax + 63) / 64, ns), dim3(64), 0, ctx->stream, S);
  CKL();
  return ORAC_OK;
}

// Up to MAX_SEGS short lists of any kinds in one launch (blockIdx.y the
// list), each with its own fixed-point accumulator, energy slots and
// dU/dlambda slot: the N1 level's 1-4 and intra-group pairs and, on M
// steps, ferrf_alchemy_add's listqq share one launch.
int small_launch_set(orac_gpu_ctx* ctx, int n, const SmallSpec* specs) {
  SmallSegs S;
  memset(&S, 0, sizeof(S));
  int ns = 0, nmax = 0;
  for (int k = 0; k < n && ns < MAX_SEGS; k++) {
    const SmallSpec& p = specs[k];
    if (p.npairs <= 0) continue;
    S.s[ns] = small_args(ctx, p.kind, p.xyz, p.pairs, p.ptype, p.npairs, p.t12, p.t6, p.fudge, p.lj_fudge,
                         p.coul_mode, 1, nullptr, p.e, p.ss, p.q, p.ffix, nullptr, p.edq);
    if (p.work && p.kind >= 3) {
      S.s[ns].lam40 = ctx->d_lam40;
      S.s[ns].work = p.work;
    }
    ns++;
    nmax = p.npairs > nmax ? p.npairs : nmax;
  }
  if (ns == 0) return ORAC_OK;
  orac_launch(k_small_segs, dim3((nmax + 63) / 64, ns), dim3(64), 0, ctx->stream, S);
  CKL();
  return ORAC_OK;
}

// fnb14_alchemy over the 1-4 list (kind 3) or ferrf_alchemy_add over listqq
// (kind 4), forces into the fixed-point accumulator, energies into d_e (4
// or 2 slots), dU/dlambda into d_edq
int alch_intra_launch(orac_gpu_ctx* ctx, int kind, const double* d_xyz, unsigned long long* d_ffix, double* d_e,
                      double* d_edq) {
  const BondedDev& B = ctx->bd;
  if (!ctx->d_lam4) return ORAC_OK;
  if (kind == 3) {
    if (B.n14 <= 0) return ORAC_OK;
    return small_launch_x(ctx, 3, d_xyz, B.p14, B.t14, B.n14, B.e1412, B.e146, B.fudge, B.lj_fudge, 1, 1, nullptr,
                          d_e, B.ss, ctx->d_aqd, d_ffix, nullptr, d_edq);
  }
  if (ctx->nlistqq <= 0) return ORAC_OK;
  return small_launch_x(ctx, 4, d_xyz, ctx->d_listqq, nullptr, ctx->nlistqq, nullptr, nullptr, 1.0, 1.0, 1, 1,
                        nullptr, d_e, B.ss, ctx->d_aqd, d_ffix, nullptr, d_edq);
}

int self_launch(orac_gpu_ctx* ctx, const int* d_ss, double* d_e) {
  orac_launch(k_self, 64, 256, 0, ctx->stream, ctx->N, ctx->d_aqd, d_ss, d_e);
  CKL();
  return ORAC_OK;
}
