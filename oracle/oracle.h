/* CPU restatement of the reference's GCMC energy hot path (FP64).
 *
 * TEST INFRASTRUCTURE: this is the oracle the GPU kernels are checked
 * against. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg load it; the product never does. Every function names the reference
 * routine it restates (paths relative to the reference project).
 *
 * Parity pin: tests/golden/ holds outputs of the reference itself (built from
 * its sources by oracle/Makefile and driven by oracle/ref_harness.c), and
 * tests/test_oracle_golden.py checks this restatement against them.
 */
#ifndef RASPA_ORACLE_H
#define RASPA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One simulation box. Orthorhombic (box[3]), or triclinic (triclinic = 1,
 * hm = the box matrix whose columns are the cell vectors, hinv its
 * inverse, both row-major): the minimum image is the rectangular or the
 * triclinic branch of ApplyBoundaryCondition (src/potentials.h:232-268). */
typedef struct {
  double box[3];
  double rc2_vdw, rc2_cc;   /* squared cut-offs */
  double overlap;           /* EnergyOverlapCriteria (src/input.c:367) */
  double coulomb;           /* COULOMBIC_CONVERSION_FACTOR (src/constants.c:162) */
  double beta;              /* 1/(k_B T) */
  int ntypes;
  const double *eps, *sig2, *shift;     /* [ntypes*ntypes] LJ table */
  int nfw;
  const double *fw_xyz;                 /* [nfw*3] */
  const int *fw_type;
  const double *fw_q;
  /* adsorbates: nmol molecules of natom atoms each, fixed stride */
  int nmol, natom, maxmol;
  double *ads_xyz;                      /* [maxmol*natom*3] */
  const int *mol_type;                  /* [natom] pseudo-atom type per atom */
  const double *mol_q;                  /* [natom] charge per atom */
  const double *mol_ref;                /* [natom*3] reference geometry */
  int start_bead;
  /* Ewald */
  int ewald;
  double alpha;
  int nk;
  const int *kidx;                      /* [nk*3] integer wave vectors */
  double *kfactor;                      /* [nk] */
  double *sk_fw, *sk_ads;               /* [nk*2] (re, im) */
  double uion, net_fw, net_ads;
  /* flexible linear chain grown from atom 0 (flexible = 1): fixed bond
   * length, harmonic bends, TraPPE torsions, LJ between atoms four or more
   * bonds apart; energies in internal units, angles in radians */
  int flexible;
  double bond, bend_k, bend_theta0, bend_sigma;
  double torsion[4], torsion_min;
  /* energy grids (UseTabularGrid, src/framework_energy.c): grid[t] != NULL
   * replaces the framework VDW pair sum of pseudo-atom type t by the lookup
   * or_grid_interpolate in that grid (plane-major, as or_grid_build writes) */
  const float *const *grid;             /* [ntypes] or NULL */
  int grid_npts[3];
  double grid_size[3], grid_shift[3], grid_cell[3];
  /* Coulomb grid of a unit probe charge (or_grid_build_coulomb): when set,
   * a bead's framework real-space charge energy is its charge times the
   * lookup (src/framework_energy.c:195-198), with no overlap test */
  const float *coul_grid;
  int coul_npts[3];
  double coul_size[3], coul_shift[3], coul_cell[3];
  /* bonded trial scheme of a flexible chain: 0 = the reference's
   * GenerateTrialOrientationsMCScheme (src/cbmc.c:1580-2480): one bend angle
   * per growth step shared by all trials, and per trial `ntors` random
   * rotations about the previous bond from which one is chosen by its
   * torsion Boltzmann factor, the chosen trial's torsion Rosenbluth factor
   * multiplying the weight (src/cbmc.c:2787-2793); 1 = bend angle and
   * dihedral drawn per trial from their Boltzmann distributions */
  int chain_scheme;
  int ntors;
  /* triclinic box */
  int triclinic;
  double hm[9], hinv[9];
  /* energy grids of a triclinic unit cell (grid_tri = 1): lookups wrap a
   * point into the unit cell through its fractional coordinates, with the
   * unit-cell matrix grid_ucm (columns a, b, c; row-major) and its inverse
   * (InterpolateVDWGrid, src/grids.c:1004-1021) */
  int grid_tri;
  double grid_ucm[9], grid_ucinv[9];
} or_sys;

/* pair terms */
double or_lj(const or_sys *s, int ta, int tb, double r2);
double or_real_ewald(const or_sys *s, double qa, double qb, double r);

/* energies of one bead at a point (no overlap logic):
 * out = {host VDW, host charge-charge, adsorbate VDW, adsorbate charge-charge}
 * (src/framework_energy.c:60,176; src/inter_energy.c:321,393) */
void or_point_energy(const or_sys *s, int type, double q, const double *p, int exclude,
                     double *out);

/* sums of |pair term| of or_point_energy (the scale of its rounding error) */
void or_point_energy_abs(const or_sys *s, int type, double q, const double *p, int exclude,
                         double *out);

/* translation/rotation energy differences for molecule m moved to new_xyz
 * (src/mc_moves.c:1601-1629 and the four *Difference routines). Returns 1 on
 * overlap; out = {dU host VDW, dU ads VDW, dU host cc, dU ads cc}. */
int or_move_delta(const or_sys *s, int m, const double *new_xyz, double *out);

/* Ewald */
void or_ewald_setup(or_sys *s);      /* kfactor, S_fw(k), UIon (src/ewald.c:532-599,615) */
void or_structure_factor(const or_sys *s, int n, const double *q, const double *xyz,
                         double *sk);
/* src/ewald.c:6859-7567: out = {dU ads-ads Fourier, dU host-ads Fourier,
 * net charge delta}; sk_new (may be NULL) receives the candidate S_ads(k). */
void or_ewald_delta(const or_sys *s, int nold, const double *xold, int nnew,
                    const double *xnew, double *out, double *sk_new);
void or_recompute_sk_ads(or_sys *s);
/* scale of or_ewald_delta's terms: out = {ads-ads, host-ads} */
void or_ewald_delta_abs(const or_sys *s, int nold, const double *xold, int nnew,
                        const double *xnew, double *out);
/* totals {host VDW, ads VDW, host cc real, ads cc real, host Fourier, ads Fourier}
 * (src/integration.c:250 CalculateEnergy for this system class) */
void or_total_energy(const or_sys *s, double *out);

/* random numbers */
typedef struct { uint64_t mt[312]; int mti; } or_mt64;
void or_mt_seed(or_mt64 *g, uint64_t seed);
double or_mt_uniform(or_mt64 *g);     /* src/utils.c:378 RandomNumber: [0,1] */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double or_philox_uniform(uint64_t seed, uint32_t system, uint64_t step, uint32_t slot);

/* random-number source for CBMC: sequential (MT) or slot-addressed (Philox) */
typedef double (*or_rng_fn)(void *ctx, int slot);
double or_rng_mt(void *ctx, int slot);

/* CBMC (src/cbmc.c). Results: out[0]=overlap, out[1]=Rosenbluth weight,
 * out[2..5]={U host VDW, U ads VDW, U host cc, U ads cc}; new_xyz receives the
 * grown positions (insertion). `exclude` is the molecule left out of the
 * adsorbate sums (nmol for an insertion). */
void or_cbmc_grow(const or_sys *s, int ntrial_first, int ntrial, or_rng_fn rng, void *ctx,
                  double *out, double *new_xyz);
void or_cbmc_retrace(const or_sys *s, int m, int ntrial_first, int ntrial, or_rng_fn rng,
                     void *ctx, double *out);

/* energy grid (src/grids.c, src/framework_hessian.c:63-109) */
void or_grid_derivatives(const or_sys *s, int type, const double *p, double *out8);
void or_grid_build(const or_sys *s, int type, const int npts[3], const double size[3],
                   const double shift[3], float *grid /* [8][nx+1][ny+1][nz+1] */);
/* CalculateDerivativesAtPositionReal (src/framework_hessian.c:111-180) for a
 * unit probe charge: out = the 8 values of or_grid_derivatives, then the
 * smallest distance to a framework atom within the cut-off */
void or_grid_derivatives_real(const or_sys *s, const double *p, double *out9);
/* the Coulomb grid (src/grids.c:586-690), layout as or_grid_build */
void or_grid_build_coulomb(const or_sys *s, const int npts[3], const double size[3], const double shift[3],
                           float *grid);
/* as or_grid_interpolate, the point wrapped into a triclinic unit cell
 * (ucm, ucinv: its matrix and inverse, row-major) when ucm is not NULL */
double or_grid_interpolate_cell(const float *grid, const int npts[3], const double size[3], const double shift[3],
                                const double cell[3], const double *ucm, const double *ucinv, const double *p);
double or_grid_interpolate(const float *grid, const int npts[3], const double size[3],
                           const double shift[3], const double cell[3], const double *p);

/* Complete GCMC engine driven by the counter-based stream that the GPU engine
 * uses. See or_mc_params. */
typedef struct {
  double cum[6];           /* cumulative move probabilities: translate, rotate, insert, delete,
                              reinsert, Widom */
  double max_translation;  /* A */
  double max_rotation;     /* rad */
  double fugacity_beta_v;  /* beta * f * V (ideal-gas Rosenbluth weight 1) */
  int ntrial_first, ntrial;
  uint64_t seed;
  uint32_t system;
} or_mc_params;

typedef struct {
  double u[6];             /* running totals as or_total_energy */
  long long attempts[6], accepted[6];   /* by move type as in cum */
  long long moves;         /* counted MC moves (see or_mc_run) */
  double widom_sum, widom_n;            /* Widom Rosenbluth weights and samples */
  double u_intra;                       /* intramolecular energy of flexible chains */
} or_mc_state;

/* intramolecular energy (bends, torsions, LJ of atoms >= 4 bonds apart) of
 * all molecules of a flexible-chain system */
double or_intra_energy(const or_sys *s);

/* Runs `nsteps` MC steps starting at step index `step0`. */
void or_mc_run(or_sys *s, const or_mc_params *p, or_mc_state *st, uint64_t step0,
               long long nsteps);

#ifdef __cplusplus
}
#endif
#endif
