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
  int kind;  // 0 fnb14, 1 fnbgrp, 2 ferrf
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
};

__device__ __forceinline__ void small_body(const SmallArgs& A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double e[4] = {0, 0, 0, 0};
  double dedl = 0.0;
  if (t < A.n) {
    const int i1 = A.pairs[2 * t] - 1, i2 = A.pairs[2 * t + 1] - 1;
    const int type = A.ss[i1] - 1;
    const double xa = A.xyz[i1] - A.xyz[i2];
    const double ya = A.xyz[A.natom + i1] - A.xyz[A.natom + i2];
    const double za = A.xyz[2 * A.natom + i1] - A.xyz[2 * A.natom + i2];
    const double rsq = xa * xa + ya * ya + za * za;
    const double rsp = sqrt(rsq);
    const double rsqi = 1.0 / rsq;
    double qforce = 0.0;
    if (A.kind == 2) {
      // ferrf: subtract fudge q q erf(alpha r)/r
      const double furpar = (A.forces ? A.fudge : 1.0) * A.q[i1] * A.q[i2];
      const double alphar = A.alpha * rsp;
      const double qt = 1.0 / (1.0 + AS_QP * alphar);
      const double expcst = exp(-alphar * alphar);
      const double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
      const double erfst = 1.0 - erfcst;
      e[type] -= furpar * erfst / rsp;
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
      e[type] += lf * (A.tab12[lij] * r12 - A.tab6[lij] * r6);
      const double furpar = qf * A.q[i1] * A.q[i2];
      if (A.coul_mode) {
        const double rspqi = rsqi / rsp;
        const double alphar = A.alpha * rsp;
        const double qt = 1.0 / (1.0 + AS_QP * alphar);
        const double expcst = exp(-alphar * alphar);
        const double erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * expcst;
        e[2 + type] += furpar * erfcst / rsp;
        qforce += furpar * (erfcst + A.twrtpi * alphar * expcst) * rspqi;
      } else {
        const double sv = furpar / rsp;
        e[2 + type] += sv;
        qforce += sv * rsqi;
      }
    }
    if (A.forces && A.ffix) {
      const double fv[3] = {qforce * xa, qforce * ya, qforce * za};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const long long q = __double2ll_rn(fv[d] * ORAC_FSCALE);
        if (q) {
          atomicAdd(A.ffix + d * A.natom + i1, (unsigned long long)q);
          atomicAdd(A.ffix + d * A.natom + i2, (unsigned long long)(-q));
        }
      }
    } else if (A.forces) {
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
  A.edq = A.dq ? d_edq : nullptr;
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
  orac_launch(k_small_segs, dim3((nmax + 255) / 256, ns), dim3(256), 0, ctx->stream, S);
  CKL();
  return ORAC_OK;
}

int self_launch(orac_gpu_ctx* ctx, const int* d_ss, double* d_e) {
  orac_launch(k_self, 64, 256, 0, ctx->stream, ctx->N, ctx->d_aqd, d_ss, d_e);
  CKL();
  return ORAC_OK;
}
