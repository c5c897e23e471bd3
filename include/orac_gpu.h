/*
 * orac_gpu.h — C ABI of the B200 implementation of ORAC's nonbonded force
 * path (liborac_gpu.so).
 *
 * The entry points replace, one for one, the Fortran routines ORAC's r-RESPA
 * driver calls on this path (file:line are positions in procacci/orac-porting):
 *
 *   orac_gpu_mts_forces       mts_forces   src/mts_forces.f:2-209
 *   orac_gpu_lc_list          lc_list      src/lc_list.f:1-237 (+ lc_index)
 *   orac_gpu_fft_pme          fft_pme      src/fft_pme.f:1-115
 *   orac_gpu_do_pmesh_kspace  do_pmesh_kspace src/pme_fftw3.f90:56-130
 *                             (argument meaning of src/pme_code.f:65-72)
 *   orac_gpu_fnb14            fnb14        src/fnb14.f:1-219
 *   orac_gpu_fnbgrp           fnbgrp       src/fnbgrp.f:1-213
 *   orac_gpu_ferrf            ferrf        src/ferrf.f:1-244
 *   orac_gpu_cself            cself        src/cself.f:1-64
 *
 * ORAC reads most inputs of these routines from Fortran module globals
 * (parst, cpropar, unit, spme).  Those are uploaded once per context with
 * orac_gpu_set_topology / _set_ewald / _set_shells / _set_box.
 *
 * Conventions (same as the Fortran arrays, so the iso_c_binding interface
 * passes them unchanged):
 *   - reals are double, integers int32; arrays are column-major;
 *   - every index stored in an array (grppt, atomp, atomg, mapnl, int14,
 *     list entries, type tables) is 1-based;
 *   - co, oc, stress, virial, recip are 3x3 column-major (a[i + 3*j] = a(i+1,j+1));
 *   - coordinates passed to mts_forces / fft_pme / lc_list are ORAC scaled box
 *     coordinates (box length 2, r = co s); do_pmesh_kspace, fnb14, fnbgrp and
 *     ferrf take Cartesian coordinates, as their Fortran counterparts do;
 *   - forces are ACCUMULATED into the caller's arrays (src/force.f:460-471);
 *     energies and the mts_forces stress are zeroed then set
 *     (src/mts_forces.f:96-107); fft_pme adds into stressc.
 *
 * Every entry point returns an int status (ORAC_OK = 0) and never aborts the
 * process; orac_gpu_last_error() gives a text for the last failure.  A context
 * owns one CUDA stream; entry points on one context are not reentrant,
 * distinct contexts may be driven from distinct host threads.
 */
#ifndef ORAC_GPU_H
#define ORAC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORAC_OK = 0,
  ORAC_ERR_PARAM = 1,    /* invalid argument or unsupported configuration */
  ORAC_ERR_CUDA = 2,     /* CUDA runtime failure */
  ORAC_ERR_CAPACITY = 3, /* list or table capacity exceeded (ORAC: xerror) */
  ORAC_ERR_STATE = 4,    /* call order violated (e.g. no topology yet) */
  ORAC_ERR_TIMEOUT = 5,  /* a device-side wait ran out of its budget */
  ORAC_ERR_NODEVICE = 6  /* no CUDA device / the library cannot run */
};

typedef struct orac_gpu_ctx orac_gpu_ctx;

/* Context life cycle ------------------------------------------------------ */
int orac_gpu_create(int device, orac_gpu_ctx** out);
int orac_gpu_destroy(orac_gpu_ctx* ctx);
const char* orac_gpu_last_error(const orac_gpu_ctx* ctx);
/* Library version and build (sm_100a) string. */
const char* orac_gpu_version(void);

/* Module globals read by mts_forces (src/mts_forces.f:120-152) and by the
 * routines it calls.  type_table is ORAC's type(ma,ma) (column-major, values
 * 1-based into ecc12/ecc6 of length ntype*(ntype+1)/2).  mapnl is the serial
 * exclusion map built by mappa (src/mappa.f): for each atom i in order,
 * [n, j_1 .. j_n] with j > i.  pmass is the mass fraction of each atom in its
 * group (ORAC's pmass/gmass, src/redmss.f:15). */
int orac_gpu_set_topology(orac_gpu_ctx* ctx, int ntap, int ngrp, int nprot,
                          const int* grppt, const int* atomp, const int* atomg,
                          const int* ss_index, const double* chrge,
                          const int* nbtype, int ntype, const int* type_table,
                          const double* ecc12, const double* ecc6,
                          const double* mass, const double* pmass,
                          double massinfty, const int* mapnl, int64_t nmapnl);

/* EWALD PME alpha n1 n2 n3 order (src/read_potential.f:133-150); clewld = 0
 * selects plain Coulomb in the real-space shells; rkcut as in blkdta.f90:386. */
int orac_gpu_set_ewald(orac_gpu_ctx* ctx, int clewld, double alphal, int order,
                       int nfft1, int nfft2, int nfft3, double rkcut);

/* r-RESPA shell radii rcut/rtol/rnei of the M, L and H shells (cpropar
 * rcutm..rneih, src/read_integrator.f:152-230).  The driver's temporary
 * swaps of these globals for the list-update calls (src/mtsmd.f:2436-2469,
 * :3287-3295) become calls to this function. */
int orac_gpu_set_shells(orac_gpu_ctx* ctx, double rcutm, double rtolm,
                        double rneim, double rcutl, double rtoll, double rneil,
                        double rcuth, double rtolh, double rneih);

/* LINKED_CELL ncx ncy ncz (src/read_potential.f:210-230). */
int orac_gpu_set_linked_cell(orac_gpu_ctx* ctx, int ncx, int ncy, int ncz);

/* Box: co (scaled -> Cartesian, upper triangular as ORAC keeps it) and its
 * inverse oc; volume = det(co) * 8. */
int orac_gpu_set_box(orac_gpu_ctx* ctx, const double* co, const double* oc);

/* lc_list: rebuild the H-shell group neighbour list from group centres
 * (scaled), radius rcut (ORAC passes rcuth+rtolh+rneih, src/mtsmd.f:2420).
 * The list stays on the device (ORAC's nnlpp0).  *npairs receives the
 * number of group pairs (may be NULL). */
int orac_gpu_lc_list(orac_gpu_ctx* ctx, double rcut, const double* xpga,
                     const double* ypga, const double* zpga, int64_t* npairs);

/* mts_forces(nstep, rshell, ...): evaluate shell rshell ('m', 'l', 'h') of
 * the standard (non-alchemical, non-REM) real-space kernel with the device
 * lists, exactly as src/mts_forces.f selects radii and lskip_ewald.  As in
 * ORAC, the 'h' call rebuilds the L list and the 'l' call the M list; a call
 * whose inner radius plus tolerance exceeds its outer radius (the phony
 * list-update calls) computes no forces.  'u' with no linked cell rebuilds
 * the H list from all pairs (src/mts_forces.f:57-65).
 * Energies: ucnp/ucns/ucnsp = LJ solute/solvent/mixed, ucop/ucos/ucosp =
 * Coulomb solute/solvent/mixed; virs, virsp are zeroed (force does not set
 * them).  Forces are accumulated into fpx/fpy/fpz, stress is set. */
int orac_gpu_mts_forces(orac_gpu_ctx* ctx, int nstep, char rshell,
                        const double* xp0, const double* yp0, const double* zp0,
                        const double* xpg, const double* ypg, const double* zpg,
                        const double* xpcm, const double* ypcm,
                        const double* zpcm, double* ucns, double* ucos,
                        double* virs, double* virsp, double* ucnp, double* ucop,
                        double* ucnsp, double* ucosp, double* fpx, double* fpy,
                        double* fpz, double* stress);

/* fft_pme (src/fft_pme.f): SPME reciprocal energy, forces and stress for
 * scaled coordinates xp and molecule centres xpcm; forces accumulated,
 * stressc accumulated (-virial + molecular correction) when pressure != 0. */
int orac_gpu_fft_pme(orac_gpu_ctx* ctx, const double* xp, const double* yp,
                     const double* zp, const double* xpcm, const double* ypcm,
                     const double* zpcm, double* eer, double* fpx, double* fpy,
                     double* fpz, double* stressc, int pressure);

/* do_pmesh_kspace: the SPME core on Cartesian coordinates with an explicit
 * recip (= 0.5 oc^T in ORAC), volume, alpha, order and grid.  dx/dy/dz are
 * accumulated, eer and virial set.  Uses the context's stream and buffers but
 * not its topology (charges are passed). */
int orac_gpu_do_pmesh_kspace(orac_gpu_ctx* ctx, int numatoms, const double* x,
                             const double* y, const double* z,
                             const double* charge, const double* recip,
                             double volume, double ewald_coeff, int order,
                             int nfft1, int nfft2, int nfft3, double* eer,
                             double* dx, double* dy, double* dz,
                             double* virial);

/* fnb14 (src/fnb14.f): 1-4 pairs int14(2,int14p), LJ tables ecc1412/ecc146
 * indexed by type14, lj_fudge and fudge; Cartesian coordinates.
 * ue[4] = LJ slt, LJ slv, Coulomb slt, Coulomb slv (set). */
int orac_gpu_fnb14(orac_gpu_ctx* ctx, const double* xp0, const double* yp0,
                   const double* zp0, int cut, const int* int14, int int14p,
                   const int* type14, const double* ecc1412,
                   const double* ecc146, int ntab, double fudge,
                   double lj_fudge, double* fpx, double* fpy, double* fpz,
                   double* ue);

/* fnbgrp (src/fnbgrp.f): non-excluded intra-group pairs ingrp(2,ingrpp);
 * Cartesian coordinates; ue[4] as fnb14. */
int orac_gpu_fnbgrp(orac_gpu_ctx* ctx, const double* xp0, const double* yp0,
                    const double* zp0, const int* ingrp, int ingrpp,
                    double* fpx, double* fpy, double* fpz, double* ue);

/* ferrf (src/ferrf.f, erf_corr off): subtract fudge*q_i q_j erf(alpha r)/r for
 * the pairs list(2,nlist); iz = 1 forces + energy, iz = 0 energy only.
 * fs[2] = (solute, solvent) energies (set). Cartesian coordinates. */
int orac_gpu_ferrf(orac_gpu_ctx* ctx, double fudge, const double* x0,
                   const double* y0, const double* z0, int iz, const int* list,
                   int nlist, double* fs, double* fpx, double* fpy,
                   double* fpz);

/* cself (src/cself.f): self energy of the context's charges. */
int orac_gpu_cself(orac_gpu_ctx* ctx, double kcut, double* self_slt,
                   double* self_slv);

/* Intramolecular terms -------------------------------------------------------
 * orac_gpu_set_bonded: the bonded terms of mts_intra_n0 / mts_intra_n1 as
 * ORAC's module arrays hold them, 1-based atoms: stretching lbnd(2, nb) with
 * r0, kb (fpbond, src/fpbond.f: U = kb (r - r0)^2); bending lbndg(3, nbend)
 * with bendpot(7, nbend) = pota..potg (fpbend, src/fpbend.f: theta0, k,
 * Urey-Bradley r0 and k, coupling terms); proper torsions ltor(4, nt) with
 * tpota = +-n, tpotb = V (fptors, src/fptors.f: U = sig (|V| - V cos n phi),
 * n = 1..8); improper torsions litr(4, nit) with ipota, ipotb, ipotc (fitors,
 * src/fitors.f: ipotc > 0 harmonic in phi, else the cosine form).  The bond
 * list is also the bond list of the erf corrections. */
int orac_gpu_set_bonded(orac_gpu_ctx* ctx, int nb, const int* lbnd,
                        const double* r0, const double* kb, int nbend,
                        const int* lbndg, const double* bendpot, int nt,
                        const int* ltor, const double* tpota,
                        const double* tpotb, int nit, const int* litr,
                        const double* ipota, const double* ipotb,
                        const double* ipotc);

/* orac_gpu_set_intra_pairs: the pair lists of mts_intra_n1 and mts_furier:
 * 1-4 pairs int14(2, n14) with type14 into the (already lj_fudge-scaled)
 * tables ecc1412/ecc146 and the Coulomb fudge (fnb14), the non-excluded
 * intra-group pairs ingrp(2, ningrp) (fnbgrp, with the topology's LJ
 * tables) and the 1-3 pairs int13(2, n13) of the erf corrections. */
int orac_gpu_set_intra_pairs(orac_gpu_ctx* ctx, int n14, const int* int14,
                             const int* type14, const double* ecc1412,
                             const double* ecc146, int ntab14, double fudge,
                             double lj_fudge, int ningrp, const int* ingrp,
                             int n13, const int* int13);

/* mts_intra_n0 (src/mts_intra_n0.f:73-100): fpbond + fpbend + fitors on
 * Cartesian coordinates; forces accumulated; energies[6] = ubond, uslvbon,
 * ubend, uslvben, uitors, uslvitor (set). */
int orac_gpu_mts_intra_n0(orac_gpu_ctx* ctx, const double* x, const double* y,
                          const double* z, double* fpx, double* fpy,
                          double* fpz, double* energies);

/* mts_intra_n1 (src/mts_intra_n1.f:76-118): fptors + fnb14 + fnbgrp;
 * forces accumulated; energies[10] = uptors, uslvtor, then the 1-4 and the
 * intra-group terms each as LJ slt, LJ slv, Coulomb slt, Coulomb slv. */
int orac_gpu_mts_intra_n1(orac_gpu_ctx* ctx, const double* x, const double* y,
                          const double* z, double* fpx, double* fpy,
                          double* fpz, double* energies);

/* Shell-kernel variants ----------------------------------------------------
 * mts_forces dispatches to force_rem, force_alchemy or force
 * (src/mts_forces.f:118-153) on the module flags rem_segment and alchemy;
 * here the context carries the flag and every later shell evaluation
 * (orac_gpu_mts_forces, _mts_forces_dev and the MD driver) uses it.
 *
 * orac_gpu_set_rem: force_rem (src/force_REM.f).  rematom[ntap] (Fortran
 * LOGICAL as int, module rem) marks the REM segment; pairs passing
 * seg_select(kind, ...) (src/rem.f90:631-645; kind 0 either atom, 1 both,
 * 2 exactly one) have their force and S'V share scaled by rem_factor(3);
 * energies stay unscaled and seg_ene (rem_hnb/lnb/mnb_energy) collects the
 * selected pairs.  rematom = NULL returns to the standard kernel. */
int orac_gpu_set_rem(orac_gpu_ctx* ctx, const int* rematom, int kind,
                     double rem_factor);
/* A new rem_factor(3) for the context's REM segment, enqueued on `stream`
 * (NULL: the context's own) so that it takes effect between steps in
 * stream order: the pair kernel reads it from device memory, so a replica
 * exchange needs no graph capture (no counterpart in the reference, whose
 * replicas keep rem_factor in a module variable). */
int orac_gpu_set_rem_factor_async(orac_gpu_ctx* ctx, double rem_factor,
                                  void* stream);

/* orac_gpu_set_alchemy: force_alchemy (src/force_alchemy.f), soft-core
 * GROMOS-like form.  ss_alchemy[ntap] (cpropar): 1 normal, 2 added, -2
 * removed (src/initialize_lambda.f:35,49); rmin, epsm per atom in internal
 * units as src/mtsmd.f:1298-1303 computes them; qsoft, ljsoft of SOFT-CORE;
 * opls selects the geometric sigma (ffield_type "opls").  Lambdas start at 0.
 * ss_alchemy = NULL returns to the standard kernel. */
int orac_gpu_set_alchemy(orac_gpu_ctx* ctx, const int* ss_alchemy,
                         const double* rmin, const double* epsm, double qsoft,
                         double ljsoft, int opls);

/* orac_gpu_set_alchemy_shift: the pair form of the alchemy variant, as
 * mts_forces selects it (src/mts_forces.f:131-146): shifted = 1 gives
 * force_ALCHEMY_shift (src/force_alchemy_shifted.f:466-520, ORAC's
 * SHIFT-POT qshift ljshift): LJ evaluated at r + ljshift 2**(1./6.) sigma
 * alch_fact(1,t) and Coulomb erfc(alpha r) / (r + qshift alch_factq(1,t));
 * shifted = 0 returns to the soft core of force_alchemy (the default).
 * Kept across orac_gpu_set_alchemy and orac_gpu_set_lambda calls. */
int orac_gpu_set_alchemy_shift(orac_gpu_ctx* ctx, int shifted, double qshift,
                               double ljshift);

/* orac_gpu_set_lambda: cpropar's ladd, lrm, laddq, lrmq and their previous
 * values ladd0..lrmq0 (lam[8] in that order), with intramol / ljintra of
 * alch_set (src/force_alchemy_shifted.f:732-790).  The PME charges become
 * (1 - |lambdaq_i|) q_i (src/mts_furier_alchemy.f:75-88).  dlam[4] (may be
 * NULL) gives d(ladd, lrm, laddq, lrmq)/dlambda of a control lambda: energy
 * evaluations then also return dU/dlambda. */
int orac_gpu_set_lambda(orac_gpu_ctx* ctx, const double* lam, int intramol,
                        int ljintra, const double* dlam);

/* Outputs of the last energy-evaluating shell call and fft_pme under a
 * variant (module globals in ORAC): out[0] seg_ene (REM), out[1] dwrk =
 * U(lambda) - U(lambda0) of the shell (src/force_alchemy.f:683-688), out[2]
 * and out[3] the LJ and Coulomb energy at lambda0, out[4] dU/dlambda of the
 * shell, out[5] the PME work eer - eer0 (src/do_pmesh_alchemy.f90:78),
 * out[6] dE_rec/dlambda of the last fft_pme (sum of the reciprocal
 * potential at each atom times its dq/dlambda), out[7] d(self energy)/dlambda
 * (cself_alchemy, src/cself_alchemy.f).  out has 8 doubles.  In MD, record
 * column 15 carries the total dU/dlambda of the window. */
int orac_gpu_variant_energies(orac_gpu_ctx* ctx, double* out);

/* Device-resident entry points -------------------------------------------
 * The same computations on device pointers (CUDA global memory, FP64 SoA),
 * for drivers that keep the state in HBM.  Forces are accumulated into the
 * device arrays fdev[0..3*ntap) laid out x|y|z; energies[8] and stress[9]
 * are device pointers that receive the shell's results (set).  energies may
 * be NULL: the shell then runs forces only and skips the FP64 pair-energy
 * evaluation (forces are identical either way). */
int orac_gpu_mts_forces_dev(orac_gpu_ctx* ctx, char rshell,
                            const double* xyz_scaled /* 3*ntap, x|y|z */,
                            const double* grp_scaled /* 3*ngrp */,
                            const double* mol_scaled /* 3*nprot */,
                            double* fdev, double* energies, double* stress);

int orac_gpu_fft_pme_dev(orac_gpu_ctx* ctx, const double* xyz_scaled,
                         const double* mol_scaled, double* fdev,
                         double* eer_dev, double* stress_dev);

/* orac_gpu_pme_kspace_static — has no counterpart in the reference.
 *
 * The SPME reciprocal sum of orac_gpu_do_pmesh_kspace for callers that cannot
 * allocate device memory: a host program that owns the HBM budget and passes
 * libraries only buffers it carved out itself, a serving loop that cannot
 * take the device-wide synchronisation cudaMalloc/cudaFree bring, a plugin
 * whose host forbids allocation.  It needs no context (creating one
 * allocates), calls no cudaMalloc, cudaFree or allocating library routine,
 * and keeps its scratch in one fixed device array of 5 MiB + 16 KiB that
 * every GPU loading the library holds until the process exits.
 *
 * Limit: each of nfft1..3 at most 256 and n1*n2*n3 at most 262144 (64^3);
 * larger grids return ORAC_ERR_CAPACITY with the reason in err.  Each axis
 * must also be at least order (2..12) and factor into 2, 3, 5, 7.
 *
 * Runs on the current device, on `stream` (a cudaStream_t; NULL = the legacy
 * default stream), asynchronously.  Device pointers: xyz[3*numatoms] Cartesian
 * x|y|z, charge[numatoms] (ORAC's internal charges), force[3*numatoms] x|y|z
 * which is ACCUMULATED into, energy[10] which receives eer then the 3x3
 * column-major virial.  recip (= 0.5 oc^T) is a host array of 9; rkcut <= 0
 * means no reciprocal-space cut.  err (may be NULL) receives a message of at
 * most err_len bytes on failure.
 *
 * Every call looks up the scratch array's device address
 * (cudaGetSymbolAddress, with the device current), so a device context that
 * is destroyed and created again (cudaDeviceReset) is followed.  The first
 * lookup on a device may load the library's device code: make the first call
 * on each device before any stream capture; a first call made while `stream`
 * is capturing returns ORAC_ERR_STATE.  Every call on a device shares the one
 * array: calls that overlap on the GPU (other streams, other host threads)
 * race and give wrong results — serialise them. */
int orac_gpu_pme_kspace_static(void* stream, int numatoms, const double* xyz,
                               const double* charge, const double* recip,
                               double volume, double ewald_coeff, double rkcut,
                               int order, int nfft1, int nfft2, int nfft3,
                               double* force, double* energy, char* err,
                               int err_len);

/* r-RESPA molecular dynamics on the device ---------------------------------
 * The NVE part of ORAC's step loop, mtsmd (src/mtsmd.f:2390-3540), with its
 * kick correc (src/correc.f), drift verlet (src/verlet.f) and the SHAKE /
 * RATTLE solvers (src/rattle_verlet.f, src/rattle_correc.f), driving the
 * shells and SPME above.  x/y/z are Cartesian positions, vx/vy/vz velocities
 * (A/fs); cnst(2,ncnst) are the rigid bonds with squared lengths dss;
 * dt_h is the outer (H) time step in fs, lrespa/mrespa/n1respa/n0respa the
 * substeps of the L, M, N1 and N0 levels, nupdte the list-update period in
 * H steps, rshk the shell ('m','l','h') that carries the SPME term; econst is
 * added to the reported total energy (self and constraint corrections).
 * The driver captures its step as CUDA graphs on the first run; a later
 * orac_gpu_set_lambda, _set_rem, _set_alchemy(_shift), _set_shells,
 * _set_ewald, _set_box or _set_linked_cell makes the next run capture them
 * again, so the change takes effect at the next step. */
int orac_gpu_md_setup(orac_gpu_ctx* ctx, const double* x, const double* y,
                      const double* z, const double* vx, const double* vy,
                      const double* vz, const int* cnst, const double* dss,
                      int ncnst, double dt_h, int lrespa, int mrespa,
                      int n1respa, int n0respa, int nupdte, char rshk,
                      double econst);

/* Advance nsteps H steps (steady-state steps run as one captured CUDA graph
 * per step kind).  Every energy_every steps one record of 16 doubles goes to
 * rec: step, kinetic, U_M LJ, U_M Coulomb, U_L LJ, U_L Coulomb, U_H LJ,
 * U_H Coulomb, E_reciprocal, econst, total, status flag, bonded (bonds,
 * bends, torsions, impropers), 1-4 + intra-group pairs, erf corrections,
 * dU/dlambda (alchemical contexts with dlam set, else 0). */
int orac_gpu_md_run(orac_gpu_ctx* ctx, int nsteps, int energy_every,
                    double* rec);

/* Queue nsteps steps on the context's stream and return at once (no energy
 * records, no status check); orac_gpu_md_collect waits, checks the status
 * (SHAKE convergence, list capacity) and gathers profiling events. */
int orac_gpu_md_run_async(orac_gpu_ctx* ctx, int nsteps);
int orac_gpu_md_collect(orac_gpu_ctx* ctx);

int orac_gpu_md_get_state(orac_gpu_ctx* ctx, double* x, double* y, double* z,
                          double* vx, double* vy, double* vz);

/* Replace positions and velocities (host arrays; pinned memory avoids a
 * staging copy).  The copies are queued on the context's stream. */
int orac_gpu_md_set_state(orac_gpu_ctx* ctx, const double* x, const double* y,
                          const double* z, const double* vx,
                          const double* vy, const double* vz);

/* 0 = launch every kernel of a step directly, 1 = replay captured graphs. */
int orac_gpu_md_set_graphs(orac_gpu_ctx* ctx, int on);

/* Energy records kept on the device.  Every energy step (md_run's
 * energy_every, or orac_gpu_batch_run_energy) writes one record of
 * 16 doubles (the layout orac_gpu_md_run returns, with [0] the
 * record's number) into a ring of the newest 2,048 records of the context.
 * Copies the newest min(max, kept) records, oldest first, to out; n_total
 * receives the number written since the last reset; reset != 0 clears the
 * count.  Column 15 holds dU/dlambda for alchemical windows
 * (orac_gpu_set_lambda with dlam), the segment energy for REM contexts and
 * the work so far under a non-equilibrium schedule, and for other contexts
 * the thermostats' energy under Nose-Hoover thermostats.  Synchronises the
 * context's stream. */
int orac_gpu_md_records(orac_gpu_ctx* ctx, int max, double* out,
                        int64_t* n_total, int reset);

/* Non-equilibrium alchemical runs (ORAC's steered alchemy, the NE work
 * swarms of test3/test4: STEER_PATH ALCHEMY with time_steer) ------------
 * orac_gpu_md_set_schedule replaces the alchemy file ORAC reads
 * (src/alchemic.f's timerec, ladded, laddedq, lremoved, lremovedq): ntimes
 * points (2..64) of increasing times in fs and the four lambdas there.
 * Call it after orac_gpu_set_alchemy and before orac_gpu_md_setup; the run
 * then starts at time t0 with the lambdas as ORAC sets them on a restart
 * (src/mtsmd.f:722-758).  Before every M shell the lambdas move to the
 * schedule's values at rtime = t0 + (N0 steps so far) x (N0 step), on the
 * device, as src/mtsmd.f:2963-2999 moves them; each M step adds ORAC's
 * work terms (src/mtsmd.f:3042-3044).  ljintra as orac_gpu_set_lambda's;
 * intramol is the last orac_gpu_set_lambda call's.  ntimes = 0 removes the
 * schedule (before the next md_setup). */
int orac_gpu_md_set_schedule(orac_gpu_ctx* ctx, int ntimes, const double* times,
                             const double* ladded, const double* laddedq,
                             const double* lremoved, const double* lremovedq,
                             double t0, int ljintra);
/* out[14]: the work so far (internal energy units), rtime (fs), ladd lrm
 * laddq lrmq, and the held terms dwrkm dwrkl dwrkh dwrkrc_m dwrkrc_l
 * dwrkrc_h dwrk_al dwrk14.  Synchronises the context's stream. */
int orac_gpu_md_work(orac_gpu_ctx* ctx, double* out);
/* (rtime, work) after each M step, the newest min(max, 8192) oldest first;
 * n_total receives the number of M steps recorded. */
int orac_gpu_md_work_trace(orac_gpu_ctx* ctx, int max, double* out,
                           int64_t* n_total);

/* Nose-Hoover thermostats (ORAC's THERMOS, NVT) ------------------------------
 * orac_gpu_md_set_thermostat replaces THERMOS / TEMPERATURE of ORAC's input
 * (src/find_thermos.f, src/cov_thermos.f): the temperature temp (K) and the
 * frequencies (cm^-1) of the three thermostats, on the molecules' centres of
 * mass, the solute atoms and the solvent atoms (ss_index 1 and 2) relative to
 * their molecule's centre of mass.  Call it before orac_gpu_md_setup; temp
 * <= 0 removes the thermostats.  The M level of every step then runs ORAC's
 * thermostat sequence (src/mtsmd.f:2556-2618, 2932, 3109-3170).  Molecules
 * whose constraints need the iterative solver (a connected set of more than
 * 4 atoms or 3 constraints) are refused at md_setup.  Energy records add
 * the thermostats' energy to the total (column 10), the extended system's
 * conserved energy, and carry it in column 15 where that column has no other
 * use (no alchemy, REM or schedule).  This replaces rank 3 of ORAC's ensembles only in part: the
 * Parrinello-Rahman barostat (ISOSTRESS, cpress) is not built. */
int orac_gpu_md_set_thermostat(orac_gpu_ctx* ctx, double temp, double nu_com,
                               double nu_solute, double nu_solvent);
/* out[13]: eta[3], etap[3] (1/fs), Q[3], ndf[3], the thermostats' energy
 * (internal units), thermostats ordered centres of mass, solute, solvent.
 * Synchronises the context's stream. */
int orac_gpu_md_thermostat(orac_gpu_ctx* ctx, double* out);
/* A restart's thermostat state (ORAC's restart records gh = eta and vh =
 * etap, src/readrs.f:247-251): eta[3] and etap[3] in the order above, after
 * orac_gpu_md_setup.  Synchronises the context's stream. */
int orac_gpu_md_set_thermostat_state(orac_gpu_ctx* ctx, const double* eta,
                                     const double* etap);

/* Batched systems ----------------------------------------------------------
 * Many independent systems (replicas, HREM states, alchemical windows), one
 * context each, advanced together: the batch splices every context's step
 * graph into one parent graph, so one launch moves all systems one H step
 * and their kernels run concurrently.  Replaces running ORAC replicas as
 * separate MPI ranks (src/rem.f90, src/orac_mpi.f90).  The contexts must be
 * set up with orac_gpu_md_setup, share one device, one list-update period
 * and one step index, and must not be driven on their own while batched.
 * The batch holds copies of the step graphs: after a parameter setter on a
 * member context, orac_gpu_batch_run returns ORAC_ERR_STATE until the batch
 * is built again. */
typedef struct orac_gpu_batch orac_gpu_batch;
int orac_gpu_batch_create(orac_gpu_ctx** ctxs, int n, orac_gpu_batch** out);
int orac_gpu_batch_run(orac_gpu_batch* b, int nsteps);
/* The same with an energy record (orac_gpu_md_records) of every system on
 * every energy_every-th step (0: none), each a captured energy step. */
int orac_gpu_batch_run_energy(orac_gpu_batch* b, int nsteps, int energy_every);
/* Every member's rem_factor(3) (factors[k] for member k), on the batch's
 * stream. */
int orac_gpu_batch_set_rem_factors(orac_gpu_batch* b, const double* factors);

/* Replica exchange: ORAC's decision (rem_exchange, src/rem.f90:371-537) for
 * n replicas over the n ensembles of a scaling ladder (ladder[e] =
 * rem_factor(3) of ensemble e).  ens[r] is the 0-based ensemble replica r
 * runs (a permutation; updated in place), pot[r] its segment energy (record
 * column 15 of its last energy step) and kT in the same units.  On
 * exchange step step_rem the pairs (p, p + 1) with p + 1 + step_rem odd
 * attempt a swap: delta = (ladder[p+1] - ladder[p]) (pot of the replica at
 * p + 1 - pot of the replica at p) / kT, accepted when delta >= 0 or
 * random <= exp(delta), one random number in [0, 1) for all pairs (ORAC's
 * broadcast one).  accepted[p] (may be NULL) is 1 where pair (p, p + 1)
 * swapped.  Host only: every rank of a multi-GPU run reaches the same
 * decision from the all-gathered energies. */
int orac_gpu_rem_exchange(int n, const double* ladder, int* ens,
                          const double* pot, double kT, long long step_rem,
                          double random, int* accepted);
int orac_gpu_batch_sync(orac_gpu_batch* b);
int orac_gpu_batch_destroy(orac_gpu_batch* b);
const char* orac_gpu_batch_last_error(const orac_gpu_batch* b);
void* orac_gpu_batch_stream(orac_gpu_batch* b);

/* Serving (no counterpart in the reference, which runs one system per
 * process, src/mtsmd.f) --------------------------------------------------
 * Executor of a request loop that keeps many systems resident on one GPU:
 * a device-memory budget (reserve / unreserve of footprints), at most
 * max_active segments in flight (the rest wait first come first served),
 * and a pump thread that launches each running segment's steps on its own
 * context stream `chunk` step graphs at a time (at most two chunks queued
 * per stream), so segments submitted while others run start at once and
 * their kernels overlap.  A context passed to submit (set up with
 * orac_gpu_md_setup) belongs to the server until poll reports its segment
 * finished; then orac_gpu_md_collect gives the run's status.  Times are
 * seconds on the host's monotonic clock (orac_gpu_server_now). */
typedef struct orac_gpu_server orac_gpu_server;
double orac_gpu_server_now(void);
int orac_gpu_server_create(int device, int64_t budget_bytes, int max_active,
                           int chunk, orac_gpu_server** out);
/* Waits for every submitted segment, stops the pump, frees the server. */
int orac_gpu_server_destroy(orac_gpu_server* s);
const char* orac_gpu_server_last_error(const orac_gpu_server* s);
/* granted = 1 and the bytes held when they fit in the budget, else 0. */
int orac_gpu_server_reserve(orac_gpu_server* s, int64_t bytes, int* granted);
int orac_gpu_server_unreserve(orac_gpu_server* s, int64_t bytes);
/* Queue a segment of nsteps H steps; t_arrival <= 0 stamps the call time. */
int orac_gpu_server_submit(orac_gpu_server* s, orac_gpu_ctx* ctx, int nsteps,
                           int64_t tag, double t_arrival, int64_t* ticket);
/* Up to max finished segments: ticket, tag, (arrival, start, end) times,
 * launch status; n = how many were returned. */
int orac_gpu_server_poll(orac_gpu_server* s, int max, int64_t* tickets,
                         int64_t* tags, double* times3, int* status, int* n);
/* pending, running, finished not yet polled, submitted, finished,
 * reserved bytes, peak reserved bytes, steps launched */
int orac_gpu_server_stats(orac_gpu_server* s, int64_t* out8);

/* Launch configuration of the real-space kernel (no counterpart in the
 * reference) ---------------------------------------------------------------
 * Lanes per i group on the M shell and on the L/H shells (16 or 32; 16 only
 * for groups of at most 4 atoms) and resident blocks per SM of its
 * forces-only build (5, 6 or 8); 0 selects the default of the context's mode
 * (alone 32, 32, 6; batched or served 16, 32, 8).  Forces, energies and
 * trajectories do not depend on it: only speed does. */
int orac_gpu_set_pair_tuning(orac_gpu_ctx* ctx, int lpg_m, int lpg_lh,
                             int minb);
/* The configuration in effect (lpg_m, lpg_lh, minb). */
int orac_gpu_get_pair_tuning(orac_gpu_ctx* ctx, int* out3);
/* Autotuner: every candidate configuration runs `trial` outer steps of the
 * context (or of the batch, all members alike) after `trial` warm-up steps,
 * timed with CUDA events; the fastest is applied, returned in out3 with its
 * time per step, and appended to the text file cache_path (may be NULL) under
 * the device name and the workload's shape (systems, atoms, group size,
 * variants).  Unless force != 0, a shape already in the file is applied
 * without timing.  The trial steps advance the systems. */
int orac_gpu_tune(orac_gpu_ctx* ctx, int trial, const char* cache_path,
                  int force, int* out3, double* ms_per_step);
int orac_gpu_batch_tune(orac_gpu_batch* b, int trial, const char* cache_path,
                        int force, int* out3, double* ms_per_step);

/* Measurement (no counterpart in the reference, which times with wall
 * clocks in src/timer.f) ---------------------------------------------------
 * The context's cudaStream_t, for callers that record their own events. */
void* orac_gpu_get_stream(orac_gpu_ctx* ctx);
/* Work counters of the real-space kernel since the last reset: list entries
 * scanned, entries kept for the next shell, atom pairs evaluated with Ewald,
 * atom pairs evaluated LJ-only. */
int orac_gpu_counters(orac_gpu_ctx* ctx, int64_t* out4, int reset);
/* Launch profiler: `on` is a mask of kernel families, bit 0 the real-space
 * pair kernel, bit 1 the integrator's drift and kick kernels, bit 2 one SPME
 * evaluation (spread to gather as one interval), bit 3 the bonded kernel
 * (on = 1 profiles the pair kernel alone).  Each launch of a profiled
 * family is bracketed by CUDA events, also inside captured graphs (a new
 * mask captures the step graphs again).  prof_read returns the pair
 * kernel's summed device time in ms and number of launches timed;
 * prof_read_family the same for family 0..3.  reset clears every family. */
int orac_gpu_prof_enable(orac_gpu_ctx* ctx, int on);
int orac_gpu_prof_read(orac_gpu_ctx* ctx, double* ms_total, int64_t* nlaunch,
                       int reset);
int orac_gpu_prof_read_family(orac_gpu_ctx* ctx, int family, double* ms_total,
                              int64_t* nlaunch, int reset);

/* FP32 FMA rate of `device` in TFLOP/s (an FMA counts 2), measured by an
 * FMA-loop kernel that fills every SM (best of three timed launches, about
 * 20 ms each); ms receives the best launch's time.  The denominator of the
 * real-space kernel's FP32 roofline. */
int orac_gpu_fp32_rate(int device, double* tflops, double* ms);

/* Bytes of device memory the context holds (every device allocation it
 * made and has not freed): the footprint a memory-budgeted scheduler
 * admits by. */
int orac_gpu_footprint(orac_gpu_ctx* ctx, int64_t* bytes);

/* Synchronise the context's stream. */
int orac_gpu_sync(orac_gpu_ctx* ctx);

/* Counters of the last calls (for measurement): number of group pairs in
 * the H/L/M lists, number of kernel launches issued by the context so far. */
int orac_gpu_stats(orac_gpu_ctx* ctx, int64_t* list_pairs /* [3] h,l,m */,
                   int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif /* ORAC_GPU_H */
