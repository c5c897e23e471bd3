// Real-space r-RESPA shell kernel: the B200 counterpart of ORAC's `force`
// (src/force.f:1-917).
//
// One warp owns one i-group (a charge group, <= ORAC_MAXG atoms, staged in
// shared memory) and its neighbour-list row.  Per partner group it
//   1. forms the group-centre minimum image in FP64 scaled coordinates and
//      classifies the pair into ORAC's bands (non-switched [rinn0, rout),
//      switched S on [rout, rout0), 1-S on [rinn, rinn0)), src/force.f:265-333;
//   2. writes the next inner shell's list entry (order preserved with a warp
//      ballot), src/force.f:279-286;
//   3. evaluates every atom pair of the two groups in FP32 -- LJ
//      ecc12/r^12 - ecc6/r^6 and q q erfc_AS(alpha r)/r with the A&S 7.1.26
//      polynomial ORAC uses -- skipping excluded pairs through the list
//      entry's mask, src/force.f:396-731;
//   4. for switched pairs adds the S'(R) V_ij term distributed by mass
//      fraction, src/force.f:754-817.
// Steps 1-2 run a lane per list entry; step 3 a lane per j atom of the
// in-band entries, queued in shared memory (k_pair below).  Forces go to
// 64-bit fixed-point accumulators with atomics, so the sum is independent
// of the order of the atomics.
// The molecular virial is assembled without per-pair work: ORAC's
// sum_pairs f (x) (Rm_i - Rm_j - img) equals sum_atoms F_a (x) Rm_a (done in
// the finalize kernel) plus, for pairs that cross the box, G_ij (x) co.img
// where G_ij is the pair's total force on the j group (done here).
#include "common.cuh"

namespace {

constexpr int WPB = 4;  // warps per block
constexpr float AS_A1 = 0.2548296f, AS_A2 = -0.28449674f, AS_A3 = 1.4214137f;
constexpr float AS_A4 = -1.453152f, AS_A5 = 1.0614054f, AS_QP = 0.3275911f;
constexpr int LJ_SMEM_MAX = 2048;  // staged LJ table entries: 16 KB beside the static queues

__device__ __forceinline__ long long to_fix(float v) { return __float2ll_rn(v * (float)ORAC_FSCALE); }

__device__ __forceinline__ void fix_add(unsigned long long* p, float v) {
  long long q = __float2ll_rn(v * (float)ORAC_FSCALE);
  if (q != 0) atomicAdd(p, (unsigned long long)q);
}

// sum over the aligned runs of W lanes of a warp
template <int W>
__device__ __forceinline__ float seg_sum(float v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of P values over the aligned runs of W lanes, scattered: at each
// shuffle step a lane keeps half of its values and receives the matching
// half of its partner's, so P - 1 shuffles (plus log2(W / P) for the last
// value) replace P full butterflies.  Returns the segment's total of value
// rs_index<W, P>(lane % W).
template <int W, int P, typename T>
__device__ __forceinline__ T reduce_scatter(T (&v)[P], int sl) {
#pragma unroll
  for (int h = P / 2, o = W / 2; h >= 1; h >>= 1, o >>= 1) {
    const bool up = (sl & o) != 0;
#pragma unroll
    for (int k = 0; k < h; k++) {
      const T send = up ? v[k] : v[k + h];
      const T keep = up ? v[k + h] : v[k];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  T r = v[0];
#pragma unroll
  for (int o = W / P / 2; o >= 1; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  return r;
}

template <int W, int P>
__device__ __forceinline__ int rs_index(int sl) {
  int idx = 0;
#pragma unroll
  for (int o = W / 2, h = P / 2; h >= 1; o >>= 1, h >>= 1) idx += (sl & o) ? h : 0;
  return idx;
}

__device__ __forceinline__ double warp_sumd(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Pair energies in FP64 from the FP64 centre distance, the stored atom
// offsets, FP64 charges and FP64 LJ parameters: used only when energies are
// requested (EN), so the FP32 force path is the same in both modes.
__device__ __forceinline__ void pair_energy_fp64(const PairArgs& A, double rx, double ry, double rz, double2 L,
                                                 bool ljon, double qq, double* conf, double* coul) {
  const double r2 = rx * rx + ry * ry + rz * rz;
  const double rsqi = 1.0 / r2;
  *conf = 0.0;
  *coul = 0.0;
  if (ljon) {
    const double r6 = rsqi * rsqi * rsqi;
    *conf = L.x * r6 * r6 - L.y * r6;
  }
  if (!A.lskip) {
    const double rsp = sqrt(r2);
    const double ar = A.alphad * rsp;
    const double qt = 1.0 / (1.0 + 0.3275911 * ar);
    const double erfcst =
        ((((1.0614054 * qt - 1.453152) * qt + 1.4214137) * qt - 0.28449674) * qt + 0.2548296) * qt * exp(-ar * ar);
    *coul = qq * erfcst / rsp;
  } else if (!A.ewald) {
    *coul = qq / sqrt(r2);
  }
}

// seg_select, src/rem.f90:631-645: 0 either atom in the segment, 1 both,
// 2 exactly one
__device__ __forceinline__ bool seg_sel(int kind, int fa, int fb) {
  const bool ra = (fa & VF_REM) != 0, rb = (fb & VF_REM) != 0;
  return kind == 0 ? (ra || rb) : (kind == 1 ? (ra && rb) : (ra != rb));
}

// Soft-core pair of force_alchemy (src/force_alchemy.f:441-531) in FP32:
// qf is the force over r, conf/coul the scaled energies that enter the S'V
// sum.  t indexes the tables (ss_i + ss_j + 4).
__device__ __forceinline__ void alch_pair_f32(const PairArgs& A, const float (*af)[9], const float (*afq)[9], float r2,
                                              int t, float rmi, float rmj, float eps4, float qq, float* qf,
                                              float* conf, float* coul) {
  if (A.at.shifted) {
    // force_ALCHEMY_shift (src/force_alchemy_shifted.f:466-520): LJ at the
    // shifted distance rl, Coulomb erfc(alpha r) over the shifted rq
    const float ir = rsqrtf(r2), r = r2 * ir;
    float f = 0.f, uc = 0.f, uq = 0.f;
    if (eps4 > 1e-12f) {
      const float sig = A.at.opls ? 2.f * sqrtf(rmi * rmj) : rmi + rmj;
      const float rl = r + A.ljshift_s * sig * af[0][t];
      const float irl = __fdividef(1.f, rl);
      const float s2 = sig * sig * irl * irl, x = s2 * s2 * s2;
      const float sc = af[1][t] * eps4;
      f = sc * (12.f * x * x - 6.f * x) * ir * irl;
      uc = sc * (x * x - x);
    }
    const float irq = __fdividef(1.f, r + A.qshift * afq[0][t]);
    if (!A.lskip) {
      const float ar = A.alphal * r;
      const float qt = __fdividef(1.0f, 1.0f + AS_QP * ar);
      const float ex = __expf(-ar * ar);
      const float erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * ex;
      const float furpar = afq[1][t] * qq;
      uq = furpar * erfcst * irq;
      // -dU/dr / r of erfc(alpha r) / rq: erfc / (r rq^2) + 2 alpha / sqrt(pi) e / (r rq)
      f += furpar * (erfcst * irq + A.twrtpi * ar * ex * ir) * irq * ir;
    } else if (!A.ewald) {
      uq = afq[1][t] * qq * irq;
      f += uq * irq * ir;
    }
    *qf = f;
    *conf = uc;
    *coul = uq;
    return;
  }
  const float auxa = rsqrtf(r2);
  const float fq1 = afq[0][t];
  const float auxaa = rsqrtf(A.qsoft * fq1 * fq1 + r2);
  float f = 0.f, uc = 0.f, uq = 0.f;
  if (eps4 > 1e-12f) {
    const float sig = A.at.opls ? 2.f * sqrtf(rmi * rmj) : rmi + rmj;
    const float s2 = sig * sig;
    const float r6 = __fdividef(r2 * r2 * r2, s2 * s2 * s2);
    const float gp1 = __fdividef(1.f, A.ljsoft * af[0][t] + r6);
    const float gp2 = gp1 * gp1;
    const float sc = af[1][t] * eps4;
    f = sc * (2.f * gp1 * gp2 - gp2) * 6.f * r6 * auxa * auxa;
    uc = sc * (gp2 - gp1);
  }
  if (!A.lskip) {
    const float rsp = r2 * auxa;
    const float ar = A.alphal * rsp;
    const float qt = __fdividef(1.0f, 1.0f + AS_QP * ar);
    const float ex = __expf(-ar * ar);
    const float erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * ex;
    const float furpar = afq[1][t] * qq;
    uq = furpar * erfcst * auxaa;
    f += uq * auxaa * auxaa + furpar * A.twrtpi * ar * ex * auxa * auxa * auxaa;
  } else if (!A.ewald) {
    uq = afq[1][t] * qq * auxaa;
    f += uq * auxaa * auxaa;
  }
  *qf = f;
  *conf = uc;
  *coul = uq;
}

// The same pair in FP64 for the energy outputs: LJ and Coulomb at lambda,
// their sum at lambda0, and dU/dlambda of the control lambda (chain rule
// through the alch_fact tables).
__device__ __forceinline__ void alch_energy_fp64(const PairArgs& A, double rx, double ry, double rz, double2 si,
                                                 double2 sj, double qq, int t, double* cd, double* qd,
                                                 double* c0, double* q0, double* du) {
  const AlchTables& T = A.at;
  const AlchDyn& D = *A.ad;
  const double rsq = rx * rx + ry * ry + rz * rz;
  if (T.shifted) {
    // force_ALCHEMY_shift's energies at lambda and lambda0, and dU/dlambda
    // through the tables: rl = r + c f0, x = (sigma/rl)^6, U = f1 e (x^2 - x),
    // dx/dlambda = -6 x c df0 / rl; Coulomb f1 g / rq, rq = r + qshift f0
    const double r = sqrt(rsq);
    const double epsmin = 4.0 * sqrt(si.y * sj.y);
    *cd = *qd = *c0 = *q0 = *du = 0.0;
    if (epsmin > 1.0e-12) {
      const double sigma = T.opls ? 2.0 * sqrt(si.x * sj.x) : si.x + sj.x;
      const double c = T.ljshift_s * sigma;
      const double rl = r + c * D.f[0][t], rl0 = r + c * D.f0[0][t];
      const double s1 = sigma / rl, s0 = sigma / rl0;
      const double x = s1 * s1 * s1 * s1 * s1 * s1, x0 = s0 * s0 * s0 * s0 * s0 * s0;
      *cd = D.f[1][t] * epsmin * (x * x - x);
      *c0 = D.f0[1][t] * epsmin * (x0 * x0 - x0);
      *du = D.df[1][t] * epsmin * (x * x - x) +
            D.f[1][t] * epsmin * (2.0 * x - 1.0) * (-6.0 * x / rl) * c * D.df[0][t];
    }
    double g = 0.0;
    if (!A.lskip) {
      const double ar = A.alphad * r;
      const double qt = 1.0 / (1.0 + 0.3275911 * ar);
      g = qq * ((((1.0614054 * qt - 1.453152) * qt + 1.4214137) * qt - 0.28449674) * qt + 0.2548296) * qt *
          exp(-ar * ar);
    } else if (!A.ewald) {
      g = qq;
    }
    if (g != 0.0) {
      const double rq = r + T.qshift * D.fq[0][t], rq0 = r + T.qshift * D.fq0[0][t];
      *qd = D.fq[1][t] * g / rq;
      *q0 = D.fq0[1][t] * g / rq0;
      *du += D.dfq[1][t] * g / rq - D.fq[1][t] * g / (rq * rq) * T.qshift * D.dfq[0][t];
    }
    return;
  }
  const double auxa = 1.0 / sqrt(rsq);
  const double fq = D.fq[0][t], fq0 = D.fq0[0][t];
  const double auxaa = 1.0 / sqrt(T.qsoft * (fq * fq) + rsq);
  const double auxa0 = 1.0 / sqrt(T.qsoft * (fq0 * fq0) + rsq);
  const double epsmin = 4.0 * sqrt(si.y * sj.y);
  *cd = *qd = *c0 = *q0 = *du = 0.0;
  if (epsmin > 1.0e-12) {
    const double sigma = T.opls ? 2.0 * sqrt(si.x * sj.x) : si.x + sj.x;
    const double s2 = sigma * sigma;
    const double r6 = rsq * rsq * rsq / (s2 * s2 * s2);
    const double gp1 = 1.0 / (T.ljsoft * D.f[0][t] + r6);
    const double gp2 = gp1 * gp1;
    const double gp10 = 1.0 / (T.ljsoft * D.f0[0][t] + r6);
    const double gp20 = gp10 * gp10;
    const double auxc = epsmin * (gp2 - gp1);
    *cd = D.f[1][t] * auxc;
    *c0 = D.f0[1][t] * epsmin * (gp20 - gp10);
    *du = D.df[1][t] * auxc + D.f[1][t] * epsmin * (gp2 - 2.0 * gp1 * gp2) * T.ljsoft * D.df[0][t];
  }
  double g = 0.0;  // charge-pair kernel without its scale and soft core
  if (!A.lskip) {
    const double ar = A.alphad / auxa;
    const double qt = 1.0 / (1.0 + 0.3275911 * ar);
    g = qq * ((((1.0614054 * qt - 1.453152) * qt + 1.4214137) * qt - 0.28449674) * qt + 0.2548296) * qt *
        exp(-ar * ar);
  } else if (!A.ewald) {
    g = qq;
  }
  if (g != 0.0) {
    *qd = D.fq[1][t] * g * auxaa;
    *q0 = D.fq0[1][t] * g * auxa0;
    *du += D.dfq[1][t] * g * auxaa - D.fq[1][t] * g * T.qsoft * fq * D.dfq[0][t] * auxaa * auxaa * auxaa;
  }
}


// Ring capacities of the per-group queues (LPG lanes own one i group).
// Entries: at most LPG - 1 left over from the previous chunk plus LPG new.
// Atom slots: at most LPG - 1 left over plus LPG entries of MG atoms.
template <int MG, int LPG>
struct Rings {
  static constexpr int QE = 2 * LPG;
  static constexpr int need = LPG - 1 + LPG * MG;
  static constexpr int QS = need <= 64 ? 64 : (need <= 128 ? 128 : (need <= 256 ? 256 : 512));
};

// A slot names one j atom of a queued entry: entry (6 bits), its position t
// among the entry's slots (3), its atom b in the j group (3), the entry's
// slot count - 1 (3).
__device__ __forceinline__ unsigned short slot_pack(int e, int t, int b, int n) {
  return (unsigned short)(e | (t << 6) | (b << 9) | ((n - 1) << 12));
}

// LPG lanes own one i group for a whole list row: 32 (a warp) for the long
// rows of the L and H lists, 16 (two groups per warp) for the short rows of
// the M list, where a full warp would leave most lanes idle.
//
// Phase 1 (a lane per list entry, LPG entries per chunk): FP64 minimum image
// and band of the group pair, the next shell's list entry, and, for an
// in-band entry, its geometry (FP32 centre distance, S, S', and in FP64 what
// the energies need) into the group's entry queue and one slot per j atom to
// evaluate into its slot queue (order kept by ballots and a segment scan).
//
// Phase 2 (a lane per j atom): passes of up to LPG slots that hold whole
// entries.  A lane takes its j atom's offset and charge once and runs over
// the i atoms (broadcast reads of shared memory): the j atom's force sums in
// the lane, and goes out with one fixed-point atomic per component, S'(R) V
// term included; the entry's V is a segmented shuffle sum over the entry's
// lanes.  The i atoms' forces sum per lane across passes and leave by one
// segment reduction at the end of the row.
//
// MINB: resident blocks per SM the forces-only build is compiled for (5, 6
// or 8; fewer registers per thread the more blocks); a context alone favours
// one launch's latency, contexts sharing the device more warps per SM.
template <int MG, bool EN, int VAR, int LPG, int MINB>
__global__ void __launch_bounds__(WPB * 32, MINB) k_pair(const PairArgs A) {
  pdl_enter();
  // the alchemy variant, and its build that also sums force_alchemy's dwrk
  constexpr bool ALCH = VAR == VAR_ALCH || VAR == VAR_ALCHW;
  constexpr int SEG = 32 / LPG;  // groups per warp
  constexpr int QE = Rings<MG, LPG>::QE, QS = Rings<MG, LPG>::QS;
  constexpr int NQ = WPB * SEG;  // groups per block
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ float2 s_lj[];
  __shared__ float4 s_ai[NQ][MG];
  __shared__ int s_ti[NQ][MG];  // the i atom's row of the LJ tables (type * ntype)
  __shared__ float s_pm[NQ][MG];
  __shared__ double s_qd[NQ][EN ? MG : 1];
  __shared__ int s_fi[NQ][VAR != VAR_STD ? MG : 1];
  __shared__ float2 s_sf[NQ][ALCH ? MG : 1];
  // entry queue: centre distance and S, S', j group metadata, skip mask;
  // FP64 distance and S and the Cartesian image for the energy build
  __shared__ float4 s_edc[NQ][QE];
  __shared__ float s_edsw[NQ][QE];
  __shared__ int2 s_emeta[NQ][QE];
  __shared__ unsigned long long s_emsk[NQ][QE];
  __shared__ double4 s_ecd[EN ? NQ : 1][EN ? QE : 1];
  __shared__ float4 s_eimg[EN ? NQ : 1][EN ? QE : 1];
  __shared__ unsigned short s_slot[NQ][QS];
  __shared__ double s_red[WPB][ACC_N];
  __shared__ double s_vimg[WPB][9];
  __shared__ float s_af[ALCH ? 2 : 1][9], s_afq[ALCH ? 2 : 1][9];

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane / LPG, sl = lane % LPG, q = warp * SEG + sub;
  const unsigned below = (1u << sl) - 1u;  // lanes of this segment below this one
  const int seg0 = sub * LPG;              // first lane of this segment
  const int nt2 = A.ntype * A.ntype;
  const bool staged = nt2 <= LJ_SMEM_MAX;
  if (threadIdx.x < WPB * 9) s_vimg[threadIdx.x / 9][threadIdx.x % 9] = 0.0;
  if (staged)
    for (int k = threadIdx.x; k < nt2; k += blockDim.x) s_lj[k] = A.lj[k];
  if constexpr (ALCH) {  // the current lambda tables
    if (threadIdx.x < 18) {
      s_af[threadIdx.x / 9][threadIdx.x % 9] = A.ad->af[threadIdx.x / 9][threadIdx.x % 9];
      s_afq[threadIdx.x / 9][threadIdx.x % 9] = A.ad->afq[threadIdx.x / 9][threadIdx.x % 9];
    }
  }
  __syncthreads();
  const float2* lj = staged ? s_lj : A.lj;
  // under lskip_ewald an atom without LJ has no pair to evaluate
  const bool ljonly = !ALCH && A.lskip && A.ewald;
  const float remf = VAR == VAR_REM ? __ldg(A.remf) : 1.f;  // rem_factor(3)
  // this segment's bits of a warp ballot
  auto segbits = [&](unsigned b) -> unsigned { return SEG == 1 ? b : (b >> seg0) & 0xffffu; };

  double ec0 = 0, ec1 = 0, ec2 = 0, eq0 = 0, eq1 = 0, eq2 = 0;
  double ex0 = 0, ex1 = 0, ex2 = 0;  // variant sums (ACC_X)
  // force_alchemy's dwrk of a forces-only launch under a schedule (A.dwrk):
  // U(lambda) - U(lambda0) of the alchemical pairs, FP64 on the FP32 pair
  // geometry (the other pairs' terms are equal at lambda and lambda0)
  double wk = 0.0;
  unsigned npairs = 0, nscan = 0, nkept = 0;
  // image term of the molecular virial: each pass's per-lane FP32 terms are
  // summed over the warp in FP64 into this warp's accumulator (stress only;
  // the terms cancel heavily, so no FP32 sums across lanes)
  float vimg[9];
#pragma unroll
  for (int c = 0; c < 9; c++) vimg[c] = 0.f;
  auto flush_vimg = [&]() {  // every lane of the warp calls it
#pragma unroll
    for (int c = 0; c < 9; c++) {
      const double t = warp_sumd((double)vimg[c]);
      if (lane == 0) s_vimg[warp][c] += t;
      vimg[c] = 0.f;
    }
  };

  // every lane of a warp runs the same trip counts, so the warp-wide
  // ballots and shuffles stay convergent
  // a row split between two warps (A.split = 2, whole-warp rows of a
  // launch that writes no next-shell list): each takes a chunk-aligned half
  // of the entries, and both add the i atoms' forces by exact fixed-point
  // atomics, so the row's result does not change; its chain is half as long
  const int split = SEG == 1 ? A.split : 1;
  for (int pw = blockIdx.x * WPB + warp; pw * SEG < A.ngrp * split; pw += gridDim.x * WPB) {
    const int gw = split == 2 ? pw >> 1 : pw;
    const int part = pw - gw * split;
    const int i = gw * SEG + sub;
    const bool gvalid = i < A.ngrp;
    const int2 mi = gvalid ? A.gmeta[i] : make_int2(0, 0);
    const int ifirst = mi.x, ni = mi.y & 0xff, typei = (mi.y >> 8) & 0xff, ljmi = mi.y >> 16;
    const double4 gi = gvalid ? A.gpos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const int row = gvalid ? A.off[i] : 0, mrow = gvalid ? A.cnt[i] : 0;
    // this warp's entries [k0, m) of the row
    const int chunk = split == 2 ? ((mrow + 1) / 2 + LPG - 1) / LPG * LPG : mrow;
    const int k0 = min(mrow, part * chunk), m = min(mrow, k0 + chunk);
    int mmax = m;
    if (SEG == 2) mmax = max(mmax, __shfl_xor_sync(FULL, m, 16));
    if (sl < ni) {
      s_ai[q][sl] = A.aoff[ifirst + sl];
      s_ti[q][sl] = A.atype[ifirst + sl] * A.ntype;
      s_pm[q][sl] = A.apm[ifirst + sl];
      if (EN) s_qd[q][sl] = A.qd[ifirst + sl];
      if (VAR != VAR_STD) s_fi[q][sl] = A.vflag[ifirst + sl];
      if (ALCH) s_sf[q][sl] = A.soft[ifirst + sl];
    }
    __syncwarp();
    // the i atoms' forces of this lane's pairs and S'V shares, in fixed
    // point: integer sums are exact, so the row's total does not depend on
    // which lane took which j atom (half or full warps, any block shape)
    long long fiq[MG][3];
#pragma unroll
    for (int a = 0; a < MG; a++) fiq[a][0] = fiq[a][1] = fiq[a][2] = 0ll;

    int nout = 0;
    int qh = 0, qn = 0;  // entry queue: head, entries pending
    int sh = 0, sn = 0;  // slot queue: head, slots pending
    for (int base = k0; base < mmax; base += LPG) {
      // ---- phase 1: geometry of list entry k (src/force.f:265-333)
      const int k = base + sl;
      const bool valid = k < m;
      int j = 0;
      unsigned long long msk = 0ull;
      int2 mj = make_int2(0, 0);
      double drj = 1e300, cx = 0.0, cy = 0.0, cz = 0.0, imx = 0.0, imy = 0.0, imz = 0.0;
      if (valid) {
        j = A.lj_[row + k];
        msk = A.lmask[row + k];
        const double4 gj = A.gpos[j];
        mj = A.gmeta[j];
        double dx = gi.x - gj.x, dy = gi.y - gj.y, dz = gi.z - gj.z;
        imx = 2.0 * round(0.5 * dx);
        imy = 2.0 * round(0.5 * dy);
        imz = 2.0 * round(0.5 * dz);
        dx -= imx;
        dy -= imy;
        dz -= imz;
        cx = A.c11 * dx + A.c12 * dy + A.c13 * dz;
        cy = A.c22 * dy + A.c23 * dz;
        cz = A.c33 * dz;
        drj = cx * cx + cy * cy + cz * cz;
      }
      if (A.next_on) {  // the next inner shell's list, order kept (src/force.f:279-286)
        const bool keep = valid && drj < A.r2neigh;
        const unsigned bal = segbits(__ballot_sync(FULL, keep));
        if (keep) {
          const int pos = nout + __popc(bal & below);
          A.j_out[row + pos] = j;
          A.mask_out[row + pos] = msk;
        }
        nout += __popc(bal);
      }
      nscan += valid ? 1u : 0u;
      if (!A.forces_on) continue;
      // band: non-switched [rinn0, rout), S on [rout, rout0), 1-S on [rinn, rinn0)
      bool inb = false;
      float sw = 1.f, dsw = 0.f;
      double swd = 1.0;
      if (valid) {
        const bool sw_out = drj >= A.r2out && drj < A.r2out0;
        const bool sw_in = drj >= A.r2inn && drj < A.r2inn0;
        inb = (drj >= A.r2inn0 && drj < A.r2out) || sw_out || sw_in;
        if (sw_out || sw_in) {
          // S(R) of src/force.f:311-317 for the forces: FP32 arithmetic on
          // the two factors taken in FP64, the distance to the band edge
          // (edge - R) and auxa (ars1 + 2R, where -3 r and 2R cancel to under
          // a tenth of their size): FP32 R would leave both with 1e-5
          // relative error.  R in FP64 from an FP32 reciprocal square root
          // and one Newton step (relative error ~1e-14); the outer band
          // gives S = auxa auxb^2, the inner one 1 - auxa auxb^2, both from
          // the same code with the band's constants.  FP64 where S enters
          // the energies.
          const double edge = sw_out ? A.rout0 : A.rinn0;
          const double ars1 = sw_out ? A.arsout1 : A.arsinn1;
          const double iars2 = sw_out ? A.diarsout2 : A.diarsinn2;
          const float iars2f = sw_out ? A.iarsout2 : A.iarsinn2;
          const float sgn = sw_out ? 1.f : -1.f;
          double y = (double)rsqrtf((float)drj);
          y = y * (1.5 - 0.5 * drj * y * y);
          const double rspd = drj * y;
          const float auxa = (float)((ars1 + 2.0 * rspd) * iars2);
          const float auxb = (float)(edge - rspd);
          const float s3 = auxa * auxb * auxb;
          sw = sw_out ? s3 : 1.0f - s3;
          dsw = sgn * (-2.0f * auxa * auxb + 2.0f * auxb * auxb * iars2f) * (float)y;
          if (EN) {
            const double auxbd = edge - rspd;
            const double s3d = (ars1 + 2.0 * rspd) * iars2 * auxbd * auxbd;
            swd = sw_out ? s3d : 1.0 - s3d;
          }
        }
      }
      // the j atoms to evaluate: all, or under lskip_ewald those with LJ --
      // and all atoms of a switched pair, which take the S'V term by mass
      // fraction whether they have LJ or not
      unsigned bm = 0u;
      if (inb) {
        bm = (1u << (mj.y & 0xff)) - 1u;
        if (ljonly && dsw == 0.f) bm &= (unsigned)(mj.y >> 16);
      }
      const int na = __popc(bm);
      int sc = na;  // inclusive scan of the slot counts over the segment
#pragma unroll
      for (int o = 1; o < LPG; o <<= 1) {
        const int v = __shfl_up_sync(FULL, sc, o);
        if (sl >= o) sc += v;
      }
      const int tot = __shfl_sync(FULL, sc, seg0 + LPG - 1);
      const unsigned bq = segbits(__ballot_sync(FULL, na > 0));
      if (na > 0) {
        const int e = (qh + qn + __popc(bq & below)) & (QE - 1);
        s_edc[q][e] = make_float4((float)cx, (float)cy, (float)cz, sw);
        s_edsw[q][e] = dsw;
        s_emeta[q][e] = mj;
        s_emsk[q][e] = msk;
        if constexpr (EN) {
          s_ecd[q][e] = make_double4(cx, cy, cz, swd);
          if (A.stress)  // j sits at its image xpg_j + img: its virial arm gains co.img
            s_eimg[q][e] = make_float4((float)(A.c11 * imx + A.c12 * imy + A.c13 * imz),
                                       (float)(A.c22 * imy + A.c23 * imz), (float)(A.c33 * imz), 0.f);
        }
        const int ps = sh + sn + sc - na;
        unsigned bb = bm;
        for (int t = 0; t < na; t++) {
          const int b = __ffs(bb) - 1;
          bb &= bb - 1u;
          s_slot[q][(ps + t) & (QS - 1)] = slot_pack(e, t, b, na);
        }
      }
      qn += __popc(bq);
      sn += tot;
      __syncwarp();

      // ---- phase 2: passes over whole entries, a lane per j atom
      const bool last = base + LPG >= m;
      for (;;) {
        const bool want = sn >= LPG || (last && sn > 0);
        if (!__any_sync(FULL, want)) break;
        int L = 0;
        if (want) {
          L = sn;
          if (sn > LPG) L = LPG - (((int)s_slot[q][(sh + LPG) & (QS - 1)] >> 6) & 7);
          else if (sn == LPG) L = LPG;
        }
        const bool act = sl < L;
        const unsigned r = act ? (unsigned)s_slot[q][(sh + sl) & (QS - 1)] : 0u;
        const int e = r & 63, t = (r >> 6) & 7, b = (r >> 9) & 7, nsl = ((r >> 12) & 7) + 1;
        float fbx = 0.f, fby = 0.f, fbz = 0.f, vpart = 0.f;
        float4 dcs = make_float4(0.f, 0.f, 0.f, 1.f);
        float dswe = 0.f;
        int jat = 0, typej = 0;
        if (act) {
          dcs = s_edc[q][e];
          dswe = s_edsw[q][e];
          const int2 me = s_emeta[q][e];
          const unsigned long long mskb = s_emsk[q][e] >> b;
          jat = me.x + b;
          typej = (me.y >> 8) & 0xff;
          const float4 ob = A.aoff[jat];
          const int tb = A.atype[jat];
          const double qbd = EN ? A.qd[jat] : 0.0;
          const int fjb = (VAR != VAR_STD) ? (int)A.vflag[jat] : 0;
          const float2 sfb = ALCH ? A.soft[jat] : make_float2(0.f, 0.f);
          const float bx = dcs.x - ob.x, by = dcs.y - ob.y, bz = dcs.z - ob.z;
          double4 cd = make_double4(0.0, 0.0, 0.0, 1.0);
          if (EN) cd = s_ecd[q][e];
          double pconf = 0.0, pcoul = 0.0, px0 = 0.0, px1 = 0.0, px2 = 0.0;
#pragma unroll
          for (int a = 0; a < MG; a++) {
            if (a >= ni) break;
            if ((mskb >> (a * 8)) & 1ull) continue;
            if (ljonly && !((ljmi >> a) & 1)) continue;
            const float4 ai = s_ai[q][a];  // a broadcast read
            const float rx = ai.x + bx, ry = ai.y + by, rz = ai.z + bz;
            float qf = 0.f, conf = 0.f, coul = 0.f;
            bool ljon = false;
            int tal = 0;
            if constexpr (ALCH) {
              // src/force_alchemy.f:412-451: exclusions and fixed-mass pairs
              // are always skipped; no LJ and no Coulomb skips the pair
              const int fia = s_fi[q][a];
              if (fia & fjb & VF_MINF) continue;
              const float2 sa = s_sf[q][a];
              const float eps4 = sa.y * sfb.y;
              if (eps4 < 1e-12f && A.lskip && A.ewald) continue;
              npairs++;
              tal = (fia >> VF_SSHIFT) + (fjb >> VF_SSHIFT) - 4;
              alch_pair_f32(A, s_af, s_afq, rx * rx + ry * ry + rz * rz, tal, sa.x, sfb.x, eps4, ai.w * ob.w, &qf, &conf,
                            &coul);
              if constexpr (VAR == VAR_ALCHW) {
                if (tal != 6) {  // 6: two normal atoms
                  double cdd, qdd, c0, q0, du;
                  alch_energy_fp64(A, (double)rx, (double)ry, (double)rz, A.softd[ifirst + a], A.softd[jat],
                                   A.qd[ifirst + a] * A.qd[jat], tal, &cdd, &qdd, &c0, &q0, &du);
                  wk += ((cdd + qdd) - (c0 + q0)) * (double)dcs.w;
                }
              }
            } else {
              const float2 Lp = lj[s_ti[q][a] + tb];
              ljon = Lp.y != 0.f;
              if (A.lskip && !ljon && A.ewald) continue;  // src/force.f:416-417
              npairs++;
              const float r2 = rx * rx + ry * ry + rz * rz;
              // 1/r from the hardware reciprocal square root, exp from ex2 and
              // an approximate reciprocal: a few ulp, far below the pair's FP32
              // rounding budget, and a fraction of the IEEE sequences' cost
              const float rinv = rsqrtf(r2);
              const float rsqi = rinv * rinv;
              if (ljon) {
                const float r6 = rsqi * rsqi * rsqi;
                const float r12 = r6 * r6;
                qf = (12.0f * Lp.x * r12 - 6.0f * Lp.y * r6) * rsqi;
                conf = Lp.x * r12 - Lp.y * r6;
              }
              if (!A.lskip) {
                const float rsp = r2 * rinv;
                const float ar = A.alphal * rsp;
                const float qt = __fdividef(1.0f, 1.0f + AS_QP * ar);
                const float ex = __expf(-ar * ar);
                const float erfcst = ((((AS_A5 * qt + AS_A4) * qt + AS_A3) * qt + AS_A2) * qt + AS_A1) * qt * ex;
                const float qq = ai.w * ob.w;
                coul = qq * erfcst * rinv;
                qf += qq * (erfcst + A.twrtpi * ar * ex) * rsqi * rinv;
              } else if (!A.ewald) {
                coul = ai.w * ob.w * rinv;
                qf += coul * rsqi;
              }
            }
            // force_rem (src/force_REM.f:491-495,634-678): selected pairs scale
            // their force and their share of the S'V sum
            const bool sel = (VAR == VAR_REM) && seg_sel(A.rem_kind, s_fi[q][a], fjb);
            vpart += sel ? (conf + coul) * remf : conf + coul;
            qf *= dcs.w;
            if (sel) qf *= remf;
            if (EN) {
              const double erx = cd.x + ((double)ai.x - (double)ob.x);
              const double ery = cd.y + ((double)ai.y - (double)ob.y);
              const double erz = cd.z + ((double)ai.z - (double)ob.z);
              double cdd, qdd;
              if constexpr (ALCH) {
                double c0, q0, du;
                alch_energy_fp64(A, erx, ery, erz, A.softd[ifirst + a], A.softd[jat], s_qd[q][a] * qbd, tal, &cdd,
                                 &qdd, &c0, &q0, &du);
                px0 += c0;
                px1 += q0;
                px2 += du;
              } else {
                pair_energy_fp64(A, erx, ery, erz, A.ljd[s_ti[q][a] + tb], ljon, s_qd[q][a] * qbd, &cdd, &qdd);
                if (sel) px0 += cdd + qdd;  // seg_ene
              }
              pconf += cdd;
              pcoul += qdd;
            }
            const float fx = qf * rx, fy = qf * ry, fz = qf * rz;
            fiq[a][0] += to_fix(fx);
            fiq[a][1] += to_fix(fy);
            fiq[a][2] += to_fix(fz);
            fbx -= fx;
            fby -= fy;
            fbz -= fz;
          }
          if constexpr (EN) {
            const int tt = typei + typej - 2;  // 0 slt-slt, 1 slt-slv, 2 slv-slv
            pconf *= cd.w;
            pcoul *= cd.w;
            if (tt == 0) {
              ec0 += pconf;
              eq0 += pcoul;
            } else if (tt == 1) {
              ec1 += pconf;
              eq1 += pcoul;
            } else {
              ec2 += pconf;
              eq2 += pcoul;
            }
            ex0 += px0 * cd.w;
            ex1 += px1 * cd.w;
            ex2 += px2 * cd.w;
          }
        }
        // S'(R) V term of switched entries (src/force.f:754-817): V summed
        // over the entry's lanes, X = -dS/dR / R V R_vec distributed by mass
        // fraction, on the j atoms here and on the i atoms at the end of the row
        if (__any_sync(FULL, dswe != 0.f)) {
          float v = vpart;
#pragma unroll
          for (int o = 1; o < MG; o <<= 1) {
            const float w = __shfl_down_sync(FULL, v, o);
            if (t + o < nsl) v += w;
          }
          const float V = __shfl_sync(FULL, v, (lane - t) & 31);
          if (act && dswe != 0.f) {
            const float sx = -dswe * V * dcs.x, sy = -dswe * V * dcs.y, sz = -dswe * V * dcs.z;
            const float pm = A.apm[jat];
            fbx -= pm * sx;
            fby -= pm * sy;
            fbz -= pm * sz;
            if (t == 0) {  // the i atoms' share, by mass fraction
#pragma unroll
              for (int a = 0; a < MG; a++) {
                if (a >= ni) break;
                const float pmi = s_pm[q][a];
                fiq[a][0] += to_fix(pmi * sx);
                fiq[a][1] += to_fix(pmi * sy);
                fiq[a][2] += to_fix(pmi * sz);
              }
            }
          }
        }
        if (act) {
          fix_add(A.ffix + jat, fbx);
          fix_add(A.ffix + A.natom + jat, fby);
          fix_add(A.ffix + 2 * A.natom + jat, fbz);
        }
        if (EN && A.stress) {
          if (act) {
            const float4 im = s_eimg[q][e];
            vimg[0] += fbx * im.x;
            vimg[1] += fbx * im.y;
            vimg[2] += fbx * im.z;
            vimg[3] += fby * im.x;
            vimg[4] += fby * im.y;
            vimg[5] += fby * im.z;
            vimg[6] += fbz * im.x;
            vimg[7] += fbz * im.y;
            vimg[8] += fbz * im.z;
          }
          flush_vimg();
        }
        const int ne = __popc(segbits(__ballot_sync(FULL, act && t == 0)));
        sh += L;
        sn -= L;
        qh += ne;
        qn -= ne;
        __syncwarp();
      }
    }
    if (A.next_on && sl == 0 && gvalid) {
      A.cnt_out[i] = nout;
      nkept += (unsigned)nout;
    }
    if (A.forces_on) {
      // i atoms: the fixed-point sums of the segment's lanes by one
      // reduce-scatter; the lane holding component c of atom a adds it
      constexpr int P = 3 * MG <= 16 ? 16 : 32;
      long long v[P];
#pragma unroll
      for (int a = 0; a < MG; a++) {
        v[3 * a] = fiq[a][0];
        v[3 * a + 1] = fiq[a][1];
        v[3 * a + 2] = fiq[a][2];
      }
#pragma unroll
      for (int k = 3 * MG; k < P; k++) v[k] = 0ll;
      const long long tot_v = reduce_scatter<LPG, P>(v, sl);
      const int idx = rs_index<LPG, P>(sl);
      const bool owner = (LPG / P <= 1) || (sl % (LPG / P)) == 0;  // one lane per value
      if (gvalid && m > 0 && owner && idx < 3 * ni && tot_v != 0)
        atomicAdd(A.ffix + (idx % 3) * A.natom + ifirst + idx / 3, (unsigned long long)tot_v);
    }
    __syncwarp();
  }
  {
    // work counters, one atomic per warp
    unsigned s0 = nscan, s1 = nkept, s2 = npairs;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(FULL, s0, o);
      s1 += __shfl_xor_sync(FULL, s1, o);
      s2 += __shfl_xor_sync(FULL, s2, o);
    }
    if (lane == 0) {
      if (s0) atomicAdd(A.wcnt + 0, (unsigned long long)s0);
      if (s1) atomicAdd(A.wcnt + 1, (unsigned long long)s1);
      if (s2) atomicAdd(A.wcnt + (A.lskip ? 3 : 2), (unsigned long long)s2);
    }
  }
  if constexpr (VAR == VAR_ALCHW) {
    const double w = warp_sumd(wk);
    if (lane == 0 && w != 0.0) atomicAdd(A.dwrk, w);
  }
  // energies and the image virial: the EN build only (a stress request
  // selects it, pair_launch)
  if (!EN || !A.forces_on) return;
  // block reduction of energies and image virial
  constexpr int NV = (VAR != VAR_STD && EN) ? 18 : 15;
  double vals[18] = {ec0, ec1, ec2, eq0, eq1, eq2, 0, 0, 0, 0, 0, 0, 0, 0, 0, ex0, ex1, ex2};
#pragma unroll
  for (int c = 0; c < NV; c++) {
    if (c >= 6 && c < 15) {
      if (lane == 0) s_red[warp][c] = s_vimg[warp][c - 6];
      continue;
    }
    const double sred = warp_sumd(vals[c]);
    if (lane == 0) s_red[warp][c] = sred;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double sacc = 0;
    for (int w = 0; w < WPB; w++) sacc += s_red[w][threadIdx.x];
    // slots 0..14 = ACC_CONF..ACC_VIMG+8, then ACC_X..ACC_X+2
    const int acc_slot = threadIdx.x < 15 ? (int)threadIdx.x : ACC_X + (int)threadIdx.x - 15;
    if (sacc != 0.0) atomicAdd(A.acc + acc_slot, sacc);
  }
}

// group centres as double4 and atom offsets from their group centre
__global__ void k_prep(int N, int G, const double* __restrict__ xyz,
                       const double* __restrict__ grp,
                       const int* __restrict__ agrp,
                       const float* __restrict__ aq, double c11, double c12,
                       double c13, double c22, double c23, double c33,
                       double4* __restrict__ gpos, float4* __restrict__ aoff,
                       unsigned long long* __restrict__ ffix) {
  pdl_enter();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < G) gpos[t] = make_double4(grp[t], grp[G + t], grp[2 * G + t], 0.0);
  if (t < N) {
    const int g = agrp[t];
    const double dx = xyz[t] - grp[g];
    const double dy = xyz[N + t] - grp[G + g];
    const double dz = xyz[2 * N + t] - grp[2 * G + g];
    aoff[t] = make_float4((float)(c11 * dx + c12 * dy + c13 * dz),
                          (float)(c22 * dy + c23 * dz), (float)(c33 * dz),
                          aq[t]);
    ffix[t] = 0ull;
    ffix[N + t] = 0ull;
    ffix[2 * N + t] = 0ull;
  }
}

// fixed point -> double forces (accumulated into fout) and the atom part of
// the molecular virial: sum_a F_a (x) co.Rm_a
__global__ void k_finalize(int N, const unsigned long long* __restrict__ ffix,
                           const double* __restrict__ mol, int P,
                           const int* __restrict__ amol, double c11, double c12,
                           double c13, double c22, double c23, double c33,
                           double* __restrict__ fout, double* __restrict__ acc) {
  pdl_enter();
  __shared__ double s_red[8][9];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (!mol) {  // forces only; the condition is uniform over the grid
    if (t < N) {
      fout[t] += (double)(long long)ffix[t] * ORAC_FSCALE_INV;
      fout[N + t] += (double)(long long)ffix[N + t] * ORAC_FSCALE_INV;
      fout[2 * N + t] += (double)(long long)ffix[2 * N + t] * ORAC_FSCALE_INV;
    }
    return;
  }
  double st[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (t < N) {
    const double fx = (double)(long long)ffix[t] * ORAC_FSCALE_INV;
    const double fy = (double)(long long)ffix[N + t] * ORAC_FSCALE_INV;
    const double fz = (double)(long long)ffix[2 * N + t] * ORAC_FSCALE_INV;
    fout[t] += fx;
    fout[N + t] += fy;
    fout[2 * N + t] += fz;
    const int p = amol[t];
    const double sx = mol[p], sy = mol[P + p], sz = mol[2 * P + p];
    const double rx = c11 * sx + c12 * sy + c13 * sz;
    const double ry = c22 * sy + c23 * sz;
    const double rz = c33 * sz;
    st[0] = fx * rx;
    st[1] = fx * ry;
    st[2] = fx * rz;
    st[3] = fy * rx;
    st[4] = fy * ry;
    st[5] = fy * rz;
    st[6] = fz * rx;
    st[7] = fz * ry;
    st[8] = fz * rz;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 9; q++) {
    const double s = warp_sumd(st[q]);
    if (lane == 0) s_red[warp][q] = s;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += s_red[w][threadIdx.x];
    atomicAdd(acc + ACC_STR + threadIdx.x, s);
  }
}

}  // namespace

int pair_launch(orac_gpu_ctx* ctx, const PairArgs& a, int maxg) {
  const size_t smem = (size_t)(a.ntype * a.ntype <= LJ_SMEM_MAX ? a.ntype * a.ntype : 0) * sizeof(float2);
  if (maxg > ORAC_MAXG)
    return ctx_fail(ctx, ORAC_ERR_PARAM, "charge group of %d atoms exceeds %d", maxg, ORAC_MAXG);
  if (a.variant < VAR_STD || a.variant > VAR_ALCH) return ctx_fail(ctx, ORAC_ERR_PARAM, "variant %d", a.variant);
  // the alchemy build that sums force_alchemy's dwrk (forces only)
  const int var = (a.variant == VAR_ALCH && a.dwrk && !a.energy && !a.stress) ? VAR_ALCHW : a.variant;
  // atoms-per-group bound of the instantiation: 3 (waters, and chains cut
  // in threes), 4, or 8; half-warp groups and the occupancy classes only
  // for the two small bounds
  const int mgk = maxg <= 3 ? 0 : (maxg <= 4 ? 1 : 2);
  const bool half = mgk < 2 && a.lpg == 16;
  const int gpb = WPB * (half ? 2 : 1);  // groups per block
  if (a.split != 1 && (a.split != 2 || half || a.next_on))
    return ctx_fail(ctx, ORAC_ERR_PARAM, "row split %d with %s", a.split, a.next_on ? "a next-shell list" : "lpg 16");
  int nb = (a.ngrp * a.split + gpb - 1) / gpb;
  if (nb < 1) nb = 1;
  int slot = -1;
  if (int rc = prof_begin(ctx, &slot)) return rc;
  const bool en = a.energy || a.stress;  // the forces-only build keeps no sums
  // occupancy class of the forces-only build: 0, 1, 2 = 5, 6, 8 blocks per SM
  const int occ = (en || mgk == 2) ? 0 : (a.minb <= 5 ? 0 : (a.minb <= 7 ? 1 : 2));
  switch ((((mgk * 4 + var) * 2 + (en ? 1 : 0)) * 2 + (half ? 1 : 0)) * 3 + occ) {
#define ORAC_KP(MGK, MG, VAR, EN, LPG, OCC, MINB)                                               \
  case (((MGK * 4 + VAR) * 2 + (EN ? 1 : 0)) * 2 + (LPG == 16 ? 1 : 0)) * 3 + OCC:             \
    orac_launch(k_pair<MG, EN, VAR, LPG, MINB>, nb, WPB * 32, smem, ctx->stream, a);            \
    break;
#define ORAC_KP_L(MGK, MG, VAR, LPG)       \
  ORAC_KP(MGK, MG, VAR, false, LPG, 0, 5)  \
  ORAC_KP(MGK, MG, VAR, false, LPG, 1, 6)  \
  ORAC_KP(MGK, MG, VAR, false, LPG, 2, 8)  \
  ORAC_KP(MGK, MG, VAR, true, LPG, 0, 1)
#define ORAC_KP_V(MGK, MG, VAR) \
  ORAC_KP_L(MGK, MG, VAR, 32)   \
  ORAC_KP_L(MGK, MG, VAR, 16)
#define ORAC_KP_W(MGK, MG)                         \
  ORAC_KP(MGK, MG, VAR_ALCHW, false, 32, 0, 5)     \
  ORAC_KP(MGK, MG, VAR_ALCHW, false, 32, 1, 6)     \
  ORAC_KP(MGK, MG, VAR_ALCHW, false, 32, 2, 8)     \
  ORAC_KP(MGK, MG, VAR_ALCHW, false, 16, 0, 5)     \
  ORAC_KP(MGK, MG, VAR_ALCHW, false, 16, 1, 6)     \
  ORAC_KP(MGK, MG, VAR_ALCHW, false, 16, 2, 8)
    ORAC_KP_V(0, 3, VAR_STD)
    ORAC_KP_V(0, 3, VAR_REM)
    ORAC_KP_V(0, 3, VAR_ALCH)
    ORAC_KP_V(1, 4, VAR_STD)
    ORAC_KP_V(1, 4, VAR_REM)
    ORAC_KP_V(1, 4, VAR_ALCH)
    ORAC_KP(2, 8, VAR_STD, false, 32, 0, 1)
    ORAC_KP(2, 8, VAR_STD, true, 32, 0, 1)
    ORAC_KP(2, 8, VAR_REM, false, 32, 0, 1)
    ORAC_KP(2, 8, VAR_REM, true, 32, 0, 1)
    ORAC_KP(2, 8, VAR_ALCH, false, 32, 0, 1)
    ORAC_KP(2, 8, VAR_ALCH, true, 32, 0, 1)
    ORAC_KP_W(0, 3)
    ORAC_KP_W(1, 4)
    ORAC_KP(2, 8, VAR_ALCHW, false, 32, 0, 1)
#undef ORAC_KP_W
#undef ORAC_KP_V
#undef ORAC_KP_L
#undef ORAC_KP
    default:
      return ctx_fail(ctx, ORAC_ERR_PARAM, "no pair-kernel build for %d atoms per group, lpg %d, %d blocks per SM",
                      maxg, a.lpg, a.minb);
  }
  CKL();
  return prof_end(ctx, slot);
}

// Inside a stream capture an event must be recorded as an external event
// node to be a real, timed record when the graph replays.
static int prof_record(orac_gpu_ctx* ctx, cudaEvent_t ev) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(ctx->stream, &cs));
  if (cs == cudaStreamCaptureStatusActive)
    CK(cudaEventRecordWithFlags(ev, ctx->stream, cudaEventRecordExternal));
  else
    CK(cudaEventRecord(ev, ctx->stream));
  return ORAC_OK;
}

int prof_begin(orac_gpu_ctx* ctx, int* slot, int family) {
  *slot = -1;
  if (!(ctx->prof & (1 << family))) return ORAC_OK;
  if (2 * (ctx->prof_next + 1) > (int)ctx->prof_ev.size()) return ORAC_OK;  // pool exhausted: not profiled
  *slot = ctx->prof_next++;
  ctx->prof_fam[*slot] = family;
  return prof_record(ctx, ctx->prof_ev[2 * *slot]);
}

int prof_end(orac_gpu_ctx* ctx, int slot) {
  if (slot < 0) return ORAC_OK;
  return prof_record(ctx, ctx->prof_ev[2 * slot + 1]);
}

int prof_collect(orac_gpu_ctx* ctx, int a, int b) {
  for (int s = a; s < b; s++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->prof_ev[2 * s], ctx->prof_ev[2 * s + 1]) != cudaSuccess) {
      cudaGetLastError();  // not sticky: mark the measurement invalid, keep running
      ctx->prof_bad = true;
      continue;
    }
    const int f = ctx->prof_fam[s];
    ctx->prof_ms[f] += ms;
    ctx->prof_n[f]++;
  }
  return ORAC_OK;
}

int prep_launch(orac_gpu_ctx* ctx, const double* xyz, const double* grp) {
  const int n = ctx->N > ctx->G ? ctx->N : ctx->G;
  const double* c = ctx->co;
  orac_launch(k_prep, (n + 255) / 256, 256, 0, ctx->stream, 
      ctx->N, ctx->G, xyz, grp, ctx->d_agrp, ctx->d_aq, c[0], c[3], c[6], c[4], c[7], c[8], ctx->d_gpos,
      ctx->d_aoff, ctx->d_ffix);
  CKL();
  return ORAC_OK;
}

int finalize_launch(orac_gpu_ctx* ctx, const double* mol, double* fout, int stress) {
  const double* c = ctx->co;
  orac_launch(k_finalize, (ctx->N + 255) / 256, 256, 0, ctx->stream, ctx->N, ctx->d_ffix, stress ? mol : nullptr, ctx->P,
                                                            ctx->d_amol, c[0], c[3], c[6], c[4], c[7], c[8], fout,
                                                            ctx->d_acc);
  CKL();
  return ORAC_OK;
}
