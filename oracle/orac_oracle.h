/*
 * ORACLE — test infrastructure only.
 *
 * FP64 CPU restatement of ORAC's nonbonded force path (procacci/orac-porting,
 * ORAC 5).  Only the tests, the smoke check and the bench's CPU-baseline leg
 * load this library, and only as the checker.  The product (liborac_gpu.so)
 * never links, loads or calls it.
 *
 * Parity status: pinned on outputs the reference printed.  The reference
 * ships no force- or energy-per-call vectors (its tests are four chaotic full
 * MD runs) and it cannot be built here (Fortran + FFTW + MPI, none
 * installed), but test2 wrote restart files at three steps of its first
 * replica and printed an energy record at each of them: the restatement,
 * given ORAC's own topology-parameter file and those restarts, reproduces the
 * records' bonded columns to the printed digits and the nonbonded and
 * reciprocal-carrying columns to 1e-4 (tests/test_oracle_orac_records.py,
 * fixtures by tests/golden/make_f0.py).  Its non-equilibrium loop reproduces
 * the lambdas of all four of test4's work files and test4's printed work at
 * 60 fs to 0.4% (tests/test_oracle_ne.py; ORAC's run is NPT).  Properties
 * the algorithm must satisfy are checked as well: forces = -dE/dx by finite
 * differences, PME against a direct Ewald k-sum, the NaCl Madelung constant,
 * the FFT against numpy.fft, and the linked-cell list against a brute-force
 * pair search.
 *
 * Conventions follow the Fortran arguments: every array is column-major,
 * every index stored in an array (grppt, atomp, mapnl, list entries, type
 * tables, bond lists) is 1-based.  co/oc/stress are 3x3 column-major
 * (co[i + 3*j] = co(i+1, j+1)).  Coordinates in force routines are ORAC
 * scaled box coordinates in [-1,1) (box length 2); PME, fnb14, fnbgrp and ferrf
 * take Cartesian coordinates, as the reference does.
 */
#ifndef ORAC_ORACLE_H
#define ORAC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* A&S 7.1.26 erfc as evaluated throughout ORAC (src/force.f:123-125,444-447). */
double orc_erfc_as(double x);

/* decide_force, src/mts_forces.f:212-241 */
int orc_decide_force(double rinn, double alphal);

/* appbou, src/appbou.f:57-69: group centres sum pmass*x */
void orc_appbou(const double* xp0, const double* yp0, const double* zp0,
                double* xpg, double* ypg, double* zpg,
                const double* pmass, int ngrp, const int* grppt);

/* change_frame, src/change_frame.f: way=1 x1 = co x0, way=-1 x1 = oc x0 */
void orc_change_frame(const double* co, const double* oc, int way, int nato,
                      const double* xp0, const double* yp0, const double* zp0,
                      double* xp1, double* yp1, double* zp1);

/* lc_index, src/lc_index.f:3-125 (+ dist_ijk, src/dist_ijk.f).
 * Returns the full-stencil count nind(2) or -1 (INDMAX overflow) or -2
 * (a cell would be visited twice: the reference stops). */
int orc_lc_index(int indmax, int ncx, int ncy, int ncz, double ctoff,
                 const double* co, int* indxi, int* indxj, int* indxk);

/* lc_list, src/lc_list.f:1-237, serial layout nnlpp = [nv, l1..lnv] per
 * group.  Returns total length written or -1 on overflow of cap. */
long orc_lc_list(int ncx, int ncy, int ncz, int nind, const int* indxi,
                 const int* indxj, const int* indxk, double rcut,
                 const double* co, const double* xp, const double* yp,
                 const double* zp, int natp, int* nnlpp, long cap);

/* force, src/force.f:1-917 (standard LJ + Ewald-erfc real-space kernel).
 * Energies are set (not accumulated); forces and stress are accumulated.
 * nnlpp/nnlpp1 use the serial layout; when rinn > 1e-5 the next inner
 * shell list is written to nnlpp1 (capacity cap1).  Returns the length of
 * nnlpp1 written (0 when none) or -1 on overflow. */
long orc_force(const int* ss_index, const double* xp0, const double* yp0,
               const double* zp0, const double* xpg, const double* ypg,
               const double* zpg, const double* charge, const int* nbtype,
               const int* type, int ma, int nato, const int* atomg,
               const double* xpcm, const double* ypcm, const double* zpcm,
               const int* atomp, const double* co, const double* ecc12,
               const double* ecc6, double alphal, const int* mapnl,
               int ngrp, const int* grppt, double* ue /* [6]: uconf slt,slv,ss
               ucoul slt,slv,ss */, double* fpx, double* fpy, double* fpz,
               double* stress, const int* nnlpp, int* nnlpp1, long cap1,
               double rneigh, double rinn, double rout, double rtolinn,
               double rtolout, const double* gmass, int iz,
               const double* mass, double massinfty, int lskip_ewald,
               int ewald, int nthreads);

/* Variants of the shell kernel selected by mts_forces (src/mts_forces.f:118-153);
 * mode 2 with `shifted` is force_ALCHEMY_shift.
 *  mode 1  force_rem (src/force_REM.f): pairs with seg_select(kind, rematom,
 *          i, j) (src/rem.f90:631-645) have their force, and their share of
 *          the S'V switching term, multiplied by rem_factor(3); the energies
 *          stay unscaled and seg_ene collects the selected pairs' LJ +
 *          Coulomb energy (switched pairs weighted by S).  In shells that skip
 *          Ewald (lskip_ewald with Ewald on) the reference adds a Coulomb term
 *          left undefined; it is taken as 0 here.
 *  mode 2  force_alchemy (src/force_alchemy.f): GROMOS-like soft core with
 *          per-atom rmin/epsm, pair class t = ss_alchemy(i) + ss_alchemy(j)
 *          in -4..4 and factor tables alch_fact(1:2, t) from alch_set
 *          (src/force_alchemy_shifted.f:732-790), for the current (fact,
 *          factq) and previous (fact0, factq0) lambdas.  Every pair in
 *          [rinn, rout0) goes through the switched loop; the work
 *          dwrk = U(lambda) - U(lambda0) (src/force_alchemy.f:683-688).
 * Tables are indexed [k][t + 4], k = 0 for alch_fact(1, t) (soft-core
 * shift), k = 1 for alch_fact(2, t) (scale). */
typedef struct {
  int mode;
  const unsigned char* rematom; /* [nato], 1 = atom of the REM segment */
  int rem_kind;                 /* 0 either, 1 both, 2 exactly one */
  double rem_factor;            /* rem_factor(3) */
  const int* ss_alchemy;        /* [nato]: 1 normal, 2 added, -2 removed */
  const double* rmin;           /* [nato] */
  const double* epsm;           /* [nato] */
  double qsoft, ljsoft;
  int opls;                     /* sigma = 2 sqrt(rmin_i rmin_j) if set */
  double fact[2][9], factq[2][9], fact0[2][9], factq0[2][9];
  /* force_ALCHEMY_shift (src/force_alchemy_shifted.f:466-520, selected by
   * mts_forces when `shifted`, src/mts_forces.f:131-138): LJ at
   * r + ljshift sigma 2^(1/6) alch_fact(1,t), Coulomb erfc(alpha r) over
   * r + qshift alch_factq(1,t), in place of the soft core */
  int shifted;
  double qshift, ljshift;
} orc_variant;

/* force with a variant (NULL or mode 0: force).  extra[4] (may be NULL)
 * receives seg_ene (mode 1), dwrk (mode 2), and the lambda0 LJ and Coulomb
 * energy totals (mode 2). */
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
                  const orc_variant* V, double* extra);

/* alch_set, src/force_alchemy_shifted.f:732-790: fact[k][t+4] for one
 * (ladd, lrm) pair; qq selects the Coulomb form of the alchemical-alchemical
 * entries. */
void orc_alch_set(double fact[2][9], double ladd, double lrm, int intramol,
                  int ljintra, int qq);

/* Bonded intramolecular forces (orac_bonded.c), Cartesian coordinates,
 * forces accumulated, ue[2] set (solute, solvent):
 * fpbond (src/fpbond.f): U = kb (r - r0)^2 over lbnd(2, nb);
 * fpbend (src/fpbend.f): pot[7 i + 0..6] = pota..potg of bend i (theta0, k,
 *   Urey-Bradley r0 and k, coupling); fptors (src/fptors.f): pota = +-n,
 *   potb = V, U = sig (|V| - V cos n phi); fitors (src/fitors.f): potc > 0
 *   harmonic in phi, else the cosine form.  fptors/fitors return the number
 *   of degenerate or unsupported terms skipped. */
void orc_fpbond(const int* ss_index, const int* lbnd, int nb, const double* x,
                const double* y, const double* z, const double* r0,
                const double* kb, double* ue, double* fx, double* fy,
                double* fz);
void orc_fpbend(const int* ss_index, const int* lbndg, int nbend,
                const double* x, const double* y, const double* z,
                const double* pot, double* ue, double* fx, double* fy,
                double* fz);
int orc_fptors(const int* ss_index, const int* ltor, int nt, const double* x,
               const double* y, const double* z, const double* pota,
               const double* potb, double* ue, double* fx, double* fy,
               double* fz);
int orc_fitors(const int* ss_index, const int* litr, int nt, const double* x,
               const double* y, const double* z, const double* pota,
               const double* potb, const double* potc, double* ue, double* fx,
               double* fy, double* fz);

/* PME (FFTW build): load_bsp_moduli + DFTMOD, src/pme_fftw3.f90:165-230 */
void orc_load_bsp_moduli(double* bsp_mod1, double* bsp_mod2, double* bsp_mod3,
                         int nfft1, int nfft2, int nfft3, int order);

/* fill_bspline, src/pme_fftw3.f90:518-576 */
void orc_fill_bspline(double w, int order, double* array, double* darray);

/* 3D transforms with FFTW's conventions for Q(n1,n2,n3) column-major:
 * r2c forward (exp(-i..)), output FQ(1+n1/2,n2,n3) interleaved complex;
 * c2r backward (exp(+i..)), unnormalised. */
void orc_fft1d(int n, double* data, int sign);
void orc_fft3d_r2c(int n1, int n2, int n3, const double* Q, double* FQ);
void orc_fft3d_c2r(int n1, int n2, int n3, const double* FQ, double* Q);

/* scalar_sum FFTW branch, src/scalar_sum.f:2-135 (in place on FQ). */
void orc_scalar_sum(double* FQ, double ewaldcof, double volume,
                    const double* recip, const double* bsp_mod1,
                    const double* bsp_mod2, const double* bsp_mod3,
                    int nfft1, int nfft2, int nfft3, double* eer, double* vir,
                    double rkcut);

/* do_pmesh_kspace FFTW branch, src/pme_fftw3.f90:56-130.
 * x,y,z Cartesian; dx,dy,dz accumulated; vir set. */
void orc_do_pmesh_kspace(int numatoms, const double* x, const double* y,
                         const double* z, const double* charge,
                         const double* recip, double volume,
                         double ewald_coeff, int order, int nfft1, int nfft2,
                         int nfft3, double* eer, double* dx, double* dy,
                         double* dz, double* vir, double rkcut, int nthreads);

/* fft_pme, src/fft_pme.f:1-115.  xp scaled, xpcm scaled; forces accumulated;
 * stressc accumulated (-vir + molecular correction) when pressure != 0. */
void orc_fft_pme(int ntap, const double* xp, const double* yp, const double* zp,
                 const double* xpcm, const double* ypcm, const double* zpcm,
                 const double* pmechg, const double* co, const double* oc,
                 double volume, double alphal, int order, int nfft1, int nfft2,
                 int nfft3, double* eer, double* fpx, double* fpy, double* fpz,
                 double* stressc, const int* atomp, int pressure, double rkcut,
                 int nthreads);

/* ferrf, src/ferrf.f:1-244 (erf_corr = .false. branches).  x Cartesian.
 * fs[2] = (slt, slv) set. iz=1 forces + energy, iz=0 energy only. */
void orc_ferrf(const int* ss_index, double alphal, const double* charge,
               double fudge, const double* x0, const double* y0,
               const double* z0, int iz, const int* list, int nlist,
               double* fs, double* fpx, double* fpy, double* fpz);

/* cself, src/cself.f:1-64 */
void orc_cself(const int* ss_index, const double* charge, int nato,
               double alphal, double kcut, double* self_slt, double* self_slv);

/* fnb14, src/fnb14.f:1-219.  ue[4] = uconf slt, slv, ucoul slt, slv (set). */
void orc_fnb14(const int* ss_index, const double* xp0, const double* yp0,
               const double* zp0, const double* charge, int nato,
               const double* ecc12, const double* ecc6, int cut, int ewald,
               double alphal, const int* int14, int int14p,
               const int* type14, double fudge, double lj_fudge, double* fpx,
               double* fpy, double* fpz, double* ue);

/* fnbgrp, src/fnbgrp.f:1-213.  ue[4] as fnb14. */
void orc_fnbgrp(const int* ss_index, const double* xp0, const double* yp0,
                const double* zp0, const double* charge, const int* type,
                const double* ecc12, const double* ecc6, int ewald,
                double alphal, const int* ingrp, int ingrpp, double* fpx,
                double* fpy, double* fpz, double* ue);

/* Oracle MD (orac_md.c): records of ORC_MD_REC = 16 doubles per energy
 * sample: step, kinetic, (LJ, Coulomb) of the M, L, H shells, SPME eer,
 * the caller's constant, total, failure flags, bonded (bonds, bends,
 * torsions, impropers), 1-4 + intra-group nonbonded, erf corrections. */
void orc_md_set_intra(void* h, int nb, const int* lbnd, const double* r0,
                      const double* kb, int nbend, const int* lbndg,
                      const double* bendpot, int nt, const int* ltor,
                      const double* tpota, const double* tpotb, int nit,
                      const int* litr, const double* ipota,
                      const double* ipotb, const double* ipotc, int n14,
                      const int* int14, const int* type14,
                      const double* ecc1412, const double* ecc146, int ntab14,
                      double fudge, int ningrp, const int* ingrp, int n13,
                      const int* int13, int n1respa, int n0respa);

/* ORAC's Nose-Hoover thermostats in the MD loop (THERMOS): temperature (K)
 * and frequencies nu[3] (cm^-1) of the centre-of-mass, solute and solvent
 * thermostats; the state out[13]: eta[3], etap[3], Q[3], ndf[3], energy. */
void orc_md_set_thermostat(void* h, double temp, const double* nu);
void orc_md_thermostat(void* h, double* out);
void orc_md_set_thermostat_state(void* h, const double* eta, const double* etap);

/* ORAC's intra-alchemical corrections (orac_oracle.c): per-atom lambdas of
 * the species, the listqq of src/initialize_lambda.f, ferrf_alchemy_add
 * (src/ferrf_alchemy_add.f) and fnb14_alchemy's Ewald branch
 * (src/fnb14_alchemy.f). */
void orc_alch_atom_lambdas(int nato, const int* ss_alchemy, double ladd, double lrm, double* lam);
int orc_alch_listqq(int nato, const int* ss_alchemy, const int* excl, int nexcl, int* out3, int cap);
void orc_ferrf_alchemy_add(const int* ss_index, double alphal, const double* charge, const double* lambdaq,
                           const double* lambdaq0, const double* x0, const double* y0, const double* z0,
                           const int* list3, int nlist, int intramol, double* fs, double* dwrk, double* fpx,
                           double* fpy, double* fpz);
void orc_fnb14_alchemy(const int* ss_index, const double* xp0, const double* yp0, const double* zp0,
                       const double* charge, const double* ecc12, const double* ecc6, double alphal,
                       const int* int14, int int14p, const int* type14, double fudge, double lj_fudge,
                       const double* lambda, const double* lambdaq, const double* lambda0, const double* lambdaq0,
                       double* fpx, double* fpy, double* fpz, double* ue, double* dwrk);

/* alchemic (src/alchemic.f), orac_md.c */
void orc_alchemic(int ntimes, const double* trec, const double* ladded, const double* laddedq,
                  const double* lremoved, const double* lremovedq, double rtime, double* g);

#ifdef __cplusplus
}
#endif

#endif
