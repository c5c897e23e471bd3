// Internal definitions shared by the translation units of liborac_gpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <utility>
#include <vector>

#include "orac_gpu.h"

// Maximum atoms per charge group handled by the pair kernel.  Exclusion and
// skip masks are stored with a fixed stride of 8 bits per i-atom.
#define ORAC_MAXG 8

// Fixed-point scale of the force accumulators: 2^40 per internal force unit
// (amu A fs^-2).  Resolution 9.1e-13, range +-8.4e6 internal units.
#define ORAC_FSCALE 1099511627776.0
#define ORAC_FSCALE_INV (1.0 / 1099511627776.0)

// Fixed-point scale of the PME charge grid: 2^40 per internal charge unit.
#define ORAC_QSCALE 1099511627776.0

// doubles per energy record of orac_gpu_md_run
#define ORAC_MD_REC 16

// Accumulator slots (double) of one force evaluation.
enum {
  ACC_CONF = 0,   // [3] LJ by type pair: slt-slt, slt-slv, slv-slv
  ACC_COUL = 3,   // [3] Coulomb by type pair
  ACC_VIMG = 6,   // [9] image term of the molecular virial, row-major
  ACC_STR = 15,   // [9] sum_a F_a (x) co.Rm_a, row-major
  ACC_X = 24,     // [3] variant sums: REM seg_ene | alchemy U0(LJ), U0(Coul), dU/dlambda
  ACC_N = 27
};

// Kernel families that the launch profiler brackets with CUDA events: the
// real-space pair kernel, the drift and kick kernels of the integrator, one
// SPME evaluation (spread to gather, as one interval), the bonded kernel.
enum { PROF_PAIR = 0, PROF_DRIFT = 1, PROF_PME = 2, PROF_BONDED = 3, PROF_NFAM = 4 };

// Shell-kernel variants, the dispatch of src/mts_forces.f:118-153.
enum { VAR_STD = 0, VAR_REM = 1, VAR_ALCH = 2 };
// the pair kernel's build of the alchemy variant that also sums
// force_alchemy's dwrk in a forces-only launch (a non-equilibrium schedule)
constexpr int VAR_ALCHW = 3;

// Per-atom variant flags (d_vflag): bit 0 REM segment atom, bit 1 mass at or
// above massinfty, bits 4..7 ss_alchemy + 4.
enum { VF_REM = 1, VF_MINF = 2, VF_SSHIFT = 4 };

// alch_fact tables of force_alchemy (src/force_alchemy.f:194-200): [k][t+4]
// with k = 0 the soft-core shift, k = 1 the scale, t = ss_i + ss_j.
struct AlchTables {
  double f[2][9], fq[2][9];    // current lambdas (LJ, Coulomb)
  double f0[2][9], fq0[2][9];  // previous lambdas
  double df[2][9], dfq[2][9];  // derivatives with respect to the control lambda
  double qsoft, ljsoft;        // SOFT-CORE parameters
  // the shifted potential of force_ALCHEMY_shift in place of the soft core
  // (SHIFT-POT qshift ljshift): Coulomb over r + qshift f, LJ at
  // r + ljshift_s sigma f, ljshift_s = ljshift 2**(1./6.) as ORAC takes it
  int shifted;
  double qshift, ljshift_s;
  int opls;                    // sigma = 2 sqrt(rmin_i rmin_j) instead of rmin_i + rmin_j
};

// The lambda-dependent tables of the alchemy variant in device memory, read
// by the pair kernel on every launch: a lambda changed on the device (a
// non-equilibrium schedule) or by orac_gpu_set_lambda needs no new graph.
// FP32 copies of the current tables for the force path, FP64 tables for
// the energies, the work and dU/dlambda.
struct AlchDyn {
  float af[2][9], afq[2][9];
  double f[2][9], fq[2][9], f0[2][9], fq0[2][9], df[2][9], dfq[2][9];
};

// A group-pair list in CSR form with fixed row capacities: row i occupies
// [off[i], off[i+1]) and holds cnt[i] entries.  Nested shell lists reuse the
// rows of their parent list.
struct GList {
  int* off = nullptr;   // [ngrp+1]
  int* cnt = nullptr;   // [ngrp]
  int* j = nullptr;     // [cap] partner group, 0-based, > row group
  unsigned long long* mask = nullptr;  // [cap] skipped atom pairs, bit a*8+b
  int64_t cap = 0;
  int64_t npairs = 0;   // host copy, updated when read back
  bool valid = false;
};

struct ShellRadii {
  double rcutm, rtolm, rneim, rcutl, rtoll, rneil, rcuth, rtolh, rneih;
};

// Arguments of one pair-kernel launch (passed by value).
struct PairArgs {
  // topology
  const double4* gpos;   // [G] scaled group centres (.w unused)
  const int2* gmeta;     // [G] (first atom, natoms | ss_type << 8)
  const float4* aoff;    // [N] Cartesian offset from group centre, charge
  const int* atype;      // [N] 0-based LJ type
  const float* apm;      // [N] mass fraction in group
  const float2* lj;      // [ntype*ntype] (ecc12, ecc6), 0 when ecc6 <= 1e-12
  int ntype;
  int ngrp;
  // box (upper triangular co)
  double c11, c12, c13, c22, c23, c33;
  // radii of this call (src/force.f:145-167)
  double r2inn, r2inn0, r2out, r2out0, rinn0, rout0, r2neigh;
  double arsout1, arsout2, arsinn1, arsinn2;
  float iarsout2, iarsinn2;  // 1/arsout2, 1/arsinn2 (0 when the band is empty)
  double diarsout2, diarsinn2;  // the same in FP64
  float alphal, twrtpi;
  double alphad;
  int forces_on, next_on, lskip, ewald;
  // energies: 0 = forces only, 1 = also FP64 pair energies
  int energy;
  const double2* ljd;  // [ntype*ntype] FP64 (ecc12, ecc6), 0 when ecc6 <= 1e-12
  const double* qd;    // [N] FP64 charges
  // lists
  const int* off;
  const int* cnt;
  const int* lj_;
  const unsigned long long* lmask;
  int* cnt_out;
  int* j_out;
  unsigned long long* mask_out;
  // outputs
  unsigned long long* ffix;  // [3N] x|y|z fixed point
  double* acc;               // [ACC_N]
  int natom;
  // work counters: list entries scanned, entries kept for the next shell,
  // atom pairs evaluated with Ewald, atom pairs evaluated LJ-only
  unsigned long long* wcnt;
  // 0: skip the image term of the molecular virial and the block reduction
  // (MD without pressure coupling needs neither)
  int stress;
  // lanes that own one i group: 32, or 16 (two groups per warp) for lists
  // with short rows; 16 applies to groups of at most 4 atoms
  int lpg;
  // resident blocks per SM of the forces-only build (5, 6 or 8)
  int minb;
  // warps per row (1, or 2 for whole-warp rows without a next-shell list)
  int split;
  // variant (VAR_*); REM: seg_select kind and rem_factor(3)
  int variant;
  const unsigned char* vflag;  // [N]
  int rem_kind;
  // rem_factor(3) in device memory: a replica exchange rewrites it without
  // capturing the step graphs again
  const float* remf;
  // alchemy: per-atom (rmin, 2 sqrt(epsm)) in FP32, (rmin, epsm) in FP64
  const float2* soft;
  const double2* softd;
  float qsoft, ljsoft;
  float qshift, ljshift_s;  // shifted potential (at.shifted)
  const AlchDyn* ad;        // the lambda tables (device memory)
  double* dwrk;             // forces-only launches under a schedule: dwrk accumulates here
  AlchTables at;            // the constants (qsoft, ljsoft, shifted, opls, shifts)
};

// Bonded intramolecular terms (orac_gpu_set_bonded / _set_intra_pairs), the
// N0 (bonds, bends, impropers) and N1 (torsions, 1-4, intra-group) terms of
// mts_intra_n0 / mts_intra_n1 and the pair lists of the erf corrections.
enum { BK_BOND = 1, BK_BEND = 2, BK_TORS = 4, BK_ITORS = 8 };
struct BondedDev {
  int nb = 0, nbend = 0, nt = 0, nit = 0;
  int2* bij = nullptr;     // 0-based atoms
  double2* bpar = nullptr;  // (r0, k)
  int4* aijk = nullptr;
  double* apot = nullptr;   // [7 nbend] pota..potg
  int4* tijkl = nullptr;
  double2* tpar = nullptr;  // (+-n, V)
  int4* iijkl = nullptr;
  double4* ipar = nullptr;  // (pota, potb, potc, 0)
  int* ss = nullptr;        // ss_index per atom
  // 1-based pair lists: 1-4 (with type14 and the scaled tables), intra-group,
  // 1-3 and bonds (for ferrf), constraints (ferrf, energy only)
  int n14 = 0, ningrp = 0, n13 = 0, ncn = 0, ntab14 = 0;
  int* p14 = nullptr;
  int* t14 = nullptr;
  double* e1412 = nullptr;
  double* e146 = nullptr;
  double fudge = 1.0, lj_fudge = 1.0;
  int* pgrp = nullptr;
  int* p13 = nullptr;
  int* pbond = nullptr;
  int* pcn = nullptr;
  int* nbt = nullptr;       // nbtype (1-based) for fnbgrp
  double* e12 = nullptr;    // LJ tables for fnbgrp
  double* e6 = nullptr;
  bool have_pairs = false;
  double* xs = nullptr;  // [6N + 16] staging of the host entry points
};

// flags of shell_run_r
enum {
  SH_ENERGY = 1,    // FP64 pair energies into the energy outputs
  SH_STRESS = 2,    // molecular virial (finalize + image term)
  SH_PREPPED = 4,   // gpos/aoff already written and the force accumulator zeroed
  SH_FIXED_OUT = 8, // d_f is a fixed-point accumulator: skip finalize
  SH_NO_NEXT = 16   // write no next-shell list (a later pass rebuilds it)
};

struct PmePlan {
  int n1 = 0, n2 = 0, n3 = 0, order = 0;
  int h1 = 0;
  float2* tw1 = nullptr;  // twiddles exp(-2 pi i k / n) per axis
  float2* tw2 = nullptr;
  float2* tw3 = nullptr;
  float* bsp1 = nullptr;  // |DFT(B-spline)|^2 moduli (double -> float)
  float* bsp2 = nullptr;
  float* bsp3 = nullptr;
  unsigned long long* qfix = nullptr;  // [n1*n2*n3] fixed-point charge grid
  float2* cgrid = nullptr;             // [h1*n2*n3] complex grid
  float* rgrid = nullptr;              // [n1*n2*n3] real grid after c2r
  float2* cgsave = nullptr;            // [h1*n2*n3] a kept transformed grid (non-equilibrium work)
  float4* theta = nullptr;             // per atom spline data cache
  int natom_cap = 0;
};

// grow-only device scratch of the short-list and SPME host entry points
struct ApiScratch {
  double* cart = nullptr;
  size_t cart_n = 0;
  double* eout = nullptr;
  int* ipairs = nullptr;
  size_t ipairs_n = 0;
  int* itype = nullptr;
  size_t itype_n = 0;
  double* t12 = nullptr;
  double* t6 = nullptr;
  size_t tab_n = 0;
  int* ss = nullptr;
  double* e4 = nullptr;
  double* q = nullptr;
  size_t q_n = 0;
};

struct MdState;  // md.cu

// A non-equilibrium alchemical run (ne.cu): the schedule as set (host) and
// the lambda state and work on the device.
constexpr int NE_MAXT = 64;       // schedule points
constexpr int NE_REC_CAP = 8192;  // (rtime, work) records, one per M step
struct NeHost {
  bool on = false;
  std::vector<double> trec, sch[4];  // times (fs); ladded laddedq lremoved lremovedq
  double t0 = 0.0;
  int ljintra = 0;
};
struct NeDev {
  int ntimes;
  double trec[NE_MAXT], sch[4][NE_MAXT];
  double t0, tn0, rtime;
  long long ninn0;     // N0 steps since t0
  double g[4], g0[4];  // ladd lrm laddq lrmq and their previous values
  double pa[4], pr[4]; // added / removed atoms: lambda, lambdaq, lambda0, lambdaq0
  int intramol, ljintra;
  double selfc;        // alpha / sqrt(pi) (1 - erfc(kcut / (2 alpha)))
  double dself;        // cself_alchemy's dwrk at the current charges
  // work terms dwrkm dwrkl dwrkh dwrkrc_m dwrkrc_l dwrkrc_h dwrk_al dwrk14:
  // held (dw) and of the evaluations of the current M step (dwn)
  double dw[8], dwn[8];
  double wrk;
  long long nrec;
  double rec[NE_REC_CAP][2];
};

// ORAC's Nose-Hoover thermostats (THERMOS): the temperature and the
// frequencies (cm^-1) of the centre-of-mass, solute and solvent thermostats,
// set before md_setup; the MD state keeps the thermostats on the device
struct ThermoHost {
  bool on = false;
  double temp = 0.0;
  double nu[3] = {0.0, 0.0, 0.0};
};

struct orac_gpu_ctx {
  MdState* md = nullptr;
  bool shared_device = false;  // advanced beside other contexts (batch, server)
  // bumped by every setter whose values kernels take by value (shells,
  // Ewald, box, cells, variant, lambdas): captured step graphs older than
  // it are captured again
  unsigned param_gen = 0;
  // pair-kernel launch configuration (orac_gpu_set_pair_tuning, the
  // autotuner): lanes per i group on the M shell and on the L/H shells,
  // resident blocks per SM; 0 = the default for the context's mode (alone:
  // 32, 32, 6; beside other contexts: 16, 32, 8).  Results do not depend on
  // it (fixed-point sums)
  int tune_lpg_m = 0, tune_lpg_lh = 0, tune_minb = 0;
  std::unordered_map<void*, size_t> dmem;  // live device allocations
  size_t dmem_bytes = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  char err[1024] = {0};
  int64_t launches = 0;

  // sizes
  int N = 0, G = 0, P = 0, ntype = 0, maxg = 0;
  bool have_topo = false, have_box = false, have_ewald = false,
       have_shells = false;

  // host copies needed by the drivers
  std::vector<int> h_gfirst, h_gn, h_amol, h_gmol;
  // atoms in a term of the intramolecular levels, bit 0 N0, bit 1 N1:
  // h_intra_b from set_bonded (bonds, bends, impropers at N0; torsions at
  // N1), h_intra_p from set_intra_pairs (1-4 and intra-group pairs at N1)
  std::vector<unsigned char> h_intra_b, h_intra_p;
  std::vector<double> h_charge, h_mass;
  std::vector<int> h_ss, h_nbtype;
  std::vector<double> h_ecc12, h_ecc6;
  ApiScratch api;

  // device topology
  int2* d_gmeta = nullptr;
  int* d_atype = nullptr;
  float* d_apm = nullptr;
  float* d_aq = nullptr;
  double* d_aqd = nullptr;
  int* d_amol = nullptr;
  int* d_agrp = nullptr;
  int* d_gmol = nullptr;
  unsigned char* d_amassinf = nullptr;
  float2* d_lj = nullptr;
  double2* d_ljd = nullptr;
  int* d_exoff = nullptr;  // [N+1]
  int* d_exj = nullptr;    // 0-based partners j > i

  // box and parameters
  double co[9] = {0}, oc[9] = {0}, volume = 0;
  ShellRadii sh{};
  int clewld = 1;
  double alphal = 0.35;
  int order = 4, nfft1 = 0, nfft2 = 0, nfft3 = 0;
  double rkcut = 1e9;
  int ncx = 0, ncy = 0, ncz = 0;
  double massinfty = 1e20;

  // per-call device buffers
  double* d_xyz = nullptr;  // [3N] scaled x|y|z
  double* d_grp = nullptr;  // [3G]
  double* d_mol = nullptr;  // [3P]
  double4* d_gpos = nullptr;
  float4* d_aoff = nullptr;
  unsigned long long* d_ffix = nullptr;  // [3N]
  double* d_acc = nullptr;               // [ACC_N]
  double* d_fout = nullptr;              // [3N] double forces of one call
  double* d_red = nullptr;               // [32] reduction scratch

  // pinned host staging
  double* h_stage = nullptr;
  size_t h_stage_bytes = 0;

  // lists: 0 = H (nnlpp0), 1 = L (nnlpp), 2 = M (nnlpp1)
  GList lists[3];
  int* d_scan_tmp = nullptr;
  int64_t* d_total = nullptr;
  int* d_flag = nullptr;

  // cell list
  int* d_cell_of = nullptr;   // [G]
  int* d_cell_cnt = nullptr;  // [ncell+1]
  int* d_cell_start = nullptr;
  int* d_cell_grp = nullptr;  // [G]
  int ncell_cap = 0;
  int* d_stencil = nullptr;   // [3*nsten]
  int nsten = 0;
  double sten_rcut = -1, sten_co[9] = {0};
  int sten_nc[3] = {0, 0, 0};

  // shell-kernel variant (orac_gpu_set_rem / orac_gpu_set_alchemy)
  int variant = VAR_STD;
  unsigned char* d_vflag = nullptr;  // [N]
  std::vector<unsigned char> h_vflag;
  int rem_kind = 0;
  double rem_factor = 1.0;
  float* d_remf = nullptr;  // [1] rem_factor on the device (the pair kernel reads it)
  float h_remf = 1.0f;      // host copy staged for orac_gpu_set_rem_factor_async
  float2* d_soft = nullptr;    // [N]
  double2* d_softd = nullptr;  // [N]
  AlchTables at{};
  BondedDev bd;
  std::vector<int> h_ssal;            // ss_alchemy
  double lam[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // ladd lrm laddq lrmq and the lambda0 set
  double* d_qc = nullptr;  // [N] PME charges at lambda: (1 - |lambdaq_i|) q_i
  double* d_q0 = nullptr;  // [N] PME charges at lambda0
  double* d_dq = nullptr;  // [N] d(PME charge)/d(control lambda), or null
  double self_dudl = 0.0;  // d(self energy)/d(control lambda) (cself_alchemy)
  // ORAC's intra-alchemical corrections (fnb14_alchemy, ferrf_alchemy_add):
  // per atom (lambda LJ, lambda charge, d(1-|lambda LJ|)/dlambda,
  // d(1-|lambda charge|)/dlambda), and listqq (ia, ib, facQ, 1-based)
  double4* d_lam4 = nullptr;
  double4* d_lam40 = nullptr;  // lambda0, lambdaq0 per atom (non-equilibrium runs)
  AlchDyn* d_ad = nullptr;  // the lambda tables the pair kernel reads
  double* pair_dwrk = nullptr;  // set around a forces-only shell whose dwrk a schedule needs
  ThermoHost thermo;         // Nose-Hoover thermostats of the MD loop (md.cu)
  NeHost ne;                 // a non-equilibrium schedule (ne.cu)
  NeDev* d_ne = nullptr;
  int4* d_ne_alist = nullptr;  // alchemical atoms: (atom, +1 added / -1 removed, ss_index, 0)
  double* d_ne_dq = nullptr;   // chrgec - chrge0 per atom
  int ne_nal = 0;
  int* d_listqq = nullptr;
  int nlistqq = -1;  // -1: not built for the current species
  int alch_intramol = 0;
  std::vector<unsigned char> h_rem;   // REM segment atoms
  bool q0_differs = false;            // lambda0 charges differ from lambda charges
  double pme_dwrk = 0.0;              // eer(lambda) - eer(lambda0) of the last fft_pme
  double* d_xtra = nullptr;  // [8] variant outputs of the last shell evaluation
  const double* pme_q() const { return variant == VAR_ALCH && d_qc ? d_qc : d_aqd; }

  // PME
  PmePlan pme;

  // measurement: work counters of the pair kernel and CUDA events around
  // its launches (recorded into captured graphs as event nodes)
  unsigned long long* d_wcnt = nullptr;  // [4]
  int prof = 0;           // mask of the profiled kernel families (PROF_*)
  bool prof_bad = false;  // an event pair could not be timed
  std::vector<cudaEvent_t> prof_ev;  // pairs (start, end)
  std::vector<int> prof_fam;         // family of each slot
  int prof_next = 0;
  double prof_ms[PROF_NFAM] = {0, 0, 0, 0};
  int64_t prof_n[PROF_NFAM] = {0, 0, 0, 0};
};

// Bumps ctx->param_gen when it goes out of scope, once armed: a setter arms
// it after its arguments have been validated, so a rejected call leaves the
// captured step graphs (and batches built on them) valid.
struct ParamGenBump {
  orac_gpu_ctx* ctx;
  bool armed = false;
  explicit ParamGenBump(orac_gpu_ctx* c) : ctx(c) {}
  void arm() { armed = true; }
  ~ParamGenBump() {
    if (armed && ctx) ctx->param_gen++;
  }
};

// record the start/end events of one profiled launch of a family (no-op
// unless that family is profiled)
int prof_begin(orac_gpu_ctx* ctx, int* slot, int family = PROF_PAIR);
int prof_end(orac_gpu_ctx* ctx, int slot);
// sum the elapsed time of slots [a, b) into prof_ms / prof_n of their
// families (after a sync)
int prof_collect(orac_gpu_ctx* ctx, int a, int b);

// shell-kernel variants (api_variant.cu)
void variant_fill(const orac_gpu_ctx* ctx, PairArgs* a);
int variant_out_launch(orac_gpu_ctx* ctx, int forces_on);
void variant_free(orac_gpu_ctx* ctx);

// ---------------------------------------------------------------- errors
int ctx_fail(orac_gpu_ctx* c, int code, const char* fmt, ...);

#define CK(call)                                                            \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                  \
      return ctx_fail(ctx, ORAC_ERR_CUDA, "%s:%d %s: %s", __FILE__,        \
                      __LINE__, #call, cudaGetErrorString(e_));             \
  } while (0)

#define CKL()                                                               \
  do {                                                                      \
    ctx->launches++;                                                        \
    cudaError_t e_ = cudaGetLastError();                                    \
    if (e_ != cudaSuccess)                                                  \
      return ctx_fail(ctx, ORAC_ERR_CUDA, "%s:%d launch: %s", __FILE__,    \
                      __LINE__, cudaGetErrorString(e_));                    \
  } while (0)

// Device allocations of a context go through dev_alloc / dev_free, which
// keep the context's footprint (bytes held on the device) for admission by
// memory budget.
static inline void dev_free(orac_gpu_ctx* ctx, void* p) {
  if (!p) return;
  auto it = ctx->dmem.find(p);
  if (it != ctx->dmem.end()) {
    ctx->dmem_bytes -= it->second;
    ctx->dmem.erase(it);
  }
  cudaFree(p);
}

template <typename T>
static inline int dev_alloc(orac_gpu_ctx* ctx, T** p, size_t n) {
  dev_free(ctx, (void*)*p);
  *p = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc((void**)p, n * sizeof(T)));
  ctx->dmem[(void*)*p] = n * sizeof(T);
  ctx->dmem_bytes += n * sizeof(T);
  return ORAC_OK;
}

// Kernel launches of the library go through orac_launch: programmatic
// dependent launch, so a kernel's blocks are scheduled while its predecessor
// in the stream still runs (in captured graphs too) and wait on the device
// for the predecessor's completion and memory (pdl_enter, the first thing
// every kernel of the library does).
template <typename... KArgs, typename... Args>
static inline cudaError_t orac_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                      cudaStream_t stream, Args&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Wait for the grids this one depends on (their memory operations complete
// and visible).  The next grid is released when this one completes: blocks
// released earlier would hold SM slots while they wait, which costs the
// concurrent systems of a batch more than it saves.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ------------------------------------------------------ internal drivers
// k_list.cu
int list_build_cells(orac_gpu_ctx* ctx, double rcut, GList* out);
int list_build_allpairs(orac_gpu_ctx* ctx, double rcut, GList* out);
int list_ensure_rows(orac_gpu_ctx* ctx, GList* L, const GList* parent);
int list_masks(orac_gpu_ctx* ctx, GList* L);
// k_pair.cu
int pair_launch(orac_gpu_ctx* ctx, const PairArgs& a, int maxg);
int prep_launch(orac_gpu_ctx* ctx, const double* xyz, const double* grp);
int finalize_launch(orac_gpu_ctx* ctx, const double* mol, double* fout_accum,
                    int stress);
// k_pme.cu
int pme_setup(orac_gpu_ctx* ctx, int n1, int n2, int n3, int order);
// d_eout[16]: energy sum (eer = 0.5 * [0]), virial sums v11 v22 v33 v12 v13
// v23 (x0.5 gives ORAC's vir), then the 9 molecular-correction terms
// row-major.  d_sxyz/d_mol may be null (no molecular correction).
int pme_run(orac_gpu_ctx* ctx, int natom, const double* d_cart /*3N*/,
            const double* d_q, const double* recip, double volume,
            double alpha, double* d_f /*3N accumulated*/, double* d_eout,
            const double* d_sxyz, const double* d_mol,
            unsigned long long* d_ffix = nullptr /*3N fixed point instead of d_f*/,
            const double* d_dq = nullptr, double* d_edq = nullptr /*sum phi_i dq_i, accumulated*/,
            float2* d_save = nullptr /*keep the transformed grid (h1 n2 n3)*/,
            const float2* d_cross = nullptr /*energy difference against a kept grid, no forces*/);
// k_small.cu: kind 0 fnb14, 1 fnbgrp, 2 ferrf; d_e[4]
int small_launch(orac_gpu_ctx* ctx, int kind, const double* d_xyz,
                 const int* d_pairs, const int* d_ptype, int npairs,
                 const double* d_t12, const double* d_t6, double fudge,
                 double lj_fudge, int coul_mode, int forces, double* d_f,
                 double* d_e, const int* d_ss);
int self_launch(orac_gpu_ctx* ctx, const int* d_ss, double* d_e);
int alch_intra_launch(orac_gpu_ctx* ctx, int kind, const double* d_xyz, unsigned long long* d_ffix, double* d_e,
                      double* d_edq);
// one short list of small_launch_set (kinds of k_small: 0 fnb14, 1 fnbgrp,
// 2 ferrf, 3 fnb14_alchemy, 4 ferrf_alchemy_add)
struct SmallSpec {
  int kind;
  const double* xyz;
  const int* pairs;
  const int* ptype;
  int npairs;
  const double* t12;
  const double* t6;
  double fudge, lj_fudge;
  int coul_mode;
  double* e;
  const int* ss;
  const double* q;
  unsigned long long* ffix;
  double* edq;
  double* work;  // fnb14_alchemy / ferrf_alchemy_add: U(lambda) - U(lambda0) (null: none)
};
int small_launch_set(orac_gpu_ctx* ctx, int n, const SmallSpec* specs);
// ne.cu: the schedule's state at md_setup, and the launches of the MD step
int ne_init(orac_gpu_ctx* ctx, double tn0);
int ne_lambda_launch(orac_gpu_ctx* ctx, int n0steps);
int ne_sum_launch(orac_gpu_ctx* ctx, int commit);
int ne_recip_launch(orac_gpu_ctx* ctx, const double* ed, const double* fq, const double* f0, int slot);
int md_nupdte(orac_gpu_ctx* ctx);
int alch_listqq_build(orac_gpu_ctx* ctx);
// the same with explicit charges (null: the topology's) and an optional
// fixed-point force output (the MD driver's level accumulators)
int small_launch_x(orac_gpu_ctx* ctx, int kind, const double* d_xyz, const int* d_pairs, const int* d_ptype,
                   int npairs, const double* d_t12, const double* d_t6, double fudge, double lj_fudge,
                   int coul_mode, int forces, double* d_f, double* d_e, const int* d_ss, const double* d_q,
                   unsigned long long* d_ffix, const double* d_dq = nullptr, double* d_edq = nullptr);
// k_small.cu: ferrf over up to four pair lists in one launch, list k with
// its own fudge, forces flag (0: energy only) and energy slots d_e[k]
int ferrf_launch_lists(orac_gpu_ctx* ctx, int nlist, const int* const* d_pairs, const int* npairs,
                       const double* fudge, const int* forces, double* const* d_e, const double* d_xyz,
                       const int* d_ss, const double* d_q, unsigned long long* d_ffix, const double* d_dq,
                       double* d_edq);
// k_bonded.cu: mask of BK_* kinds; forces into d_f (FP64 atomics) or d_ffix
// (fixed point; the proper torsions into d_ffix_tors when given, so one
// launch serves two r-RESPA levels); d_e[8] (bond, bend, tors, itors) x
// (slt, slv) or null
int bonded_launch(orac_gpu_ctx* ctx, int mask, const double* d_x, double* d_f, unsigned long long* d_ffix,
                  double* d_e, unsigned long long* d_ffix_tors = nullptr);
void bonded_free(orac_gpu_ctx* ctx);
int bonded_set_constraints(orac_gpu_ctx* ctx, const int* cnst, int ncnst);
// api.cu
int shell_run(orac_gpu_ctx* ctx, char rshell, const double* d_xyz,
              const double* d_grp, const double* d_mol, double* d_f,
              double* d_e, double* d_stress, int energy);
// the same with explicit shell radii (the driver's list-update calls swap
// radii, src/mtsmd.f:2436-2469)
int shell_run_r(orac_gpu_ctx* ctx, char rshell, const ShellRadii& radii,
                const double* d_xyz, const double* d_grp, const double* d_mol,
                double* d_f, double* d_e, double* d_stress, int energy);
// graph-capturable H-list rebuild: no host synchronisation, capacity must be
// reserved beforehand; an overflow sets *d_flag bit 1 and leaves the list
// invalid on the device
int list_build_cells_async(orac_gpu_ctx* ctx, double rcut, GList* out,
                           int* d_flag);
int list_prepare_stencil(orac_gpu_ctx* ctx, double rcut);
// md.cu
void md_destroy(orac_gpu_ctx* ctx);
// device part of fft_pme (api_pme.cu)
int fft_pme_device(orac_gpu_ctx* ctx, const double* d_sxyz,
                   const double* d_mol, double* d_f, double* d_eout);
