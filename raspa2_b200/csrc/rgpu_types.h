/* Host/device shared layouts of the B200 GCMC energy path.
 *
 * One `RgpuSys` describes one simulation box: geometry, force-field tables
 * resolved for the adsorbate component, Ewald constants, MC move parameters
 * and the device pointers of the box's state. It is built on the host
 * (capi.cu) and copied to device memory; kernels copy it into shared memory.
 *
 * Positions on the mixed-precision path are 32-bit fixed-point fractional
 * coordinates: x_fix = round(frac(x / L) * 2^32) as a signed int. The
 * difference of two such ints, taken with wrap-around, is the minimum-image
 * separation in units of L / 2^32, so the periodic boundary condition of
 * ApplyBoundaryCondition (src/potentials.h:241-245) costs one integer
 * subtraction and the separation keeps 24 significant bits relative to its
 * own length rather than to the box length. (Valid for orthorhombic boxes at
 * least twice the cut-off, which the reference also requires.)
 */
#ifndef RGPU_TYPES_H
#define RGPU_TYPES_H

#include <stdint.h>

#define RGPU_MAX_ATOMS 8       /* atoms per adsorbate molecule */
#define RGPU_MAX_FWTYPES 4     /* framework pseudo-atom types */
#define RGPU_MAX_TRIALS 16     /* CBMC trial positions per step */
#define RGPU_MAX_POS 64        /* bead positions evaluated in one batch */
#define RGPU_MAX_TORS 128      /* torsion candidates per chain trial (chain_scheme 0; the reference default is 100) */
#define RGPU_TILE 16           /* framework atoms per tile (mixed-precision layout) */

/* per-system counters */
enum {
  RGPU_CNT_ATTEMPT = 0,  /* [0..3]: translation, rotation, insertion, deletion */
  RGPU_CNT_ACCEPT = 4,   /* [4..7] */
  RGPU_CNT_MOVES = 8,    /* counted MC moves */
  RGPU_CNT_OVERLAP = 9,  /* proposals rejected by overlap */
  RGPU_CNT_PAIRS = 10,   /* bead-atom pairs visited */
  RGPU_CNT_INCUT = 11,   /* pairs inside the cut-off (LJ evaluated) */
  RGPU_CNT_CHARGED = 12, /* of those, pairs with a real-space charge term */
  RGPU_CNT_KSITES = 13,  /* wave vector x site products of dS(k) */
  RGPU_CNT_KVEC = 14,    /* wave vectors summed (energy terms) */
  RGPU_CNT_CYCLES = 15,  /* SM clock cycles the system spent in the engine */
  RGPU_CNT_CYC_EVAL = 16, /* of those, in pair-energy evaluations (rank 0) */
  RGPU_CNT_CYC_EWALD = 17, /* of those, in Ewald sums (rank 0) */
  RGPU_CNT_REINS_ATTEMPT = 18, /* CBMC reinsertions attempted */
  RGPU_CNT_REINS_ACCEPT = 19,  /* and accepted */
  RGPU_NCNT = 20
};

/* per-system running energies (internal units, FP64) */
enum {
  RGPU_E_HOST_VDW = 0, RGPU_E_ADS_VDW = 1, RGPU_E_HOST_REAL = 2, RGPU_E_ADS_REAL = 3,
  RGPU_E_HOST_FOURIER = 4, RGPU_E_ADS_FOURIER = 5,
  RGPU_E_INTRA = 6,      /* bend + torsion + intramolecular LJ of flexible molecules */
  RGPU_NE = 8
};

/* status word bits */
enum {
  RGPU_OK = 0,
  RGPU_ERR_MAXMOL = 1,      /* an insertion was refused for lack of molecule slots */
  RGPU_ERR_NONFINITE = 2,   /* a non-finite energy reached an acceptance test */
};

/* per-system sums for ensemble averages, over the steps at or after
 * RgpuState.step[2] */
enum {
  RGPU_SUM_SAMPLES = 0,  /* steps sampled */
  RGPU_SUM_N = 1,        /* molecules */
  RGPU_SUM_N2 = 2,
  RGPU_SUM_U = 3,        /* total energy (the six running terms) */
  RGPU_SUM_UN = 4,
  RGPU_SUM_U2 = 5,
  RGPU_SUM_WIDOM_W = 6,  /* Widom test insertions: sum of Rosenbluth weights */
  RGPU_SUM_WIDOM_N = 7,  /* and their number */
  RGPU_NSUM = 8
};

/* The mutable state of one system in device memory, one block so that the
 * host reads it with one copy. */
typedef struct {
  double energy[RGPU_NE];            /* running energies */
  long long counters[RGPU_NCNT];
  double sums[RGPU_NSUM];
  /* [0] next step index, [1] step at which the engine stops advancing this
   * system (exclusive), [2] first step entering the sums, [3] unused */
  unsigned long long step[4];
  int nmol;
  int status;
  int pad[2];
} RgpuState;

typedef struct {
  double eps4, sig2, shift;   /* 4*epsilon, sigma^2, U(rc) */
} RgpuLJ;

typedef struct {
  float eps4, sig2, shift, pad;
} RgpuLJf;

/* Tile of the mixed-precision framework layout: RGPU_TILE spatially close atoms.
 * c = centre in fixed point with the atom count in .w; h = half extents (A)
 * such that every atom of the tile lies within +-h of c (minimum image). */
typedef struct {
  int4 c;
  float4 h;
} TileRec;

/* geometry of an energy grid: npts cells per axis over `size` from `shift`,
 * spanning a unit cell of lengths `cell`; a triclinic unit cell (tri = 1)
 * has its matrix (columns a, b, c; row-major) and then its inverse in
 * device memory at uc[0..17] */
typedef struct {
  int npts[3];
  int tri;
  double size[3], shift[3], cell[3];
  const double *uc;
} RgpuGridGeom;

typedef struct RgpuSys {
  /* geometry */
  double box[3], inv_box[3];
  float fix_scale[3];         /* L / 2^32 per axis */
  /* triclinic box (triclinic = 1): hm = box matrix (columns a, b, c),
   * hinv its inverse, row-major; hmf = hm / 2^32 in FP32 (Cartesian
   * difference from fixed-point fractional differences); wperp = the
   * perpendicular widths (distance between opposite faces) */
  int triclinic;
  float wperp[3];
  double hm[9], hinv[9];
  float hmf[9];
  float rc2f;
  double rc2;                 /* VDW and real-space cut-off squared (equal) */
  double overlap;             /* EnergyOverlapCriteria */
  double beta;
  double coulomb, alpha;
  float coulombf, alphaf;
  /* framework, sorted by pseudo-atom type into segments */
  int nfw;
  int nseg;
  int seg_start[RGPU_MAX_FWTYPES + 1];
  int fw_charged;             /* any framework charge != 0 */
  /* adsorbate component */
  int natom, start_bead, maxmol;
  int mol_charged;
  double mol_q[RGPU_MAX_ATOMS];
  float mol_qf[RGPU_MAX_ATOMS];
  double mol_ref[RGPU_MAX_ATOMS][3];
  RgpuLJ lj_bf[RGPU_MAX_ATOMS][RGPU_MAX_FWTYPES];   /* bead atom x framework segment */
  RgpuLJ lj_bb[RGPU_MAX_ATOMS][RGPU_MAX_ATOMS];     /* bead atom x bead atom */
  RgpuLJf ljf_bf[RGPU_MAX_ATOMS][RGPU_MAX_FWTYPES];
  RgpuLJf ljf_bb[RGPU_MAX_ATOMS][RGPU_MAX_ATOMS];
  /* Ewald (charges only) */
  int ewald, nk;
  int kmax[3];
  double self_mol;            /* sum over the molecule's sites of K q^2 alpha / sqrt(pi) */
  double excl_mol;            /* intramolecular exclusion energy of the rigid molecule (reference geometry) */
  double uion, net_fw, mol_charge;
  /* MC */
  double cum[6];              /* cumulative move probabilities (order of rgpu_system_desc.move_cum) */
  double max_translation, max_rotation;
  double fugacity_beta_v;     /* beta * f * V, ideal-gas Rosenbluth weight 1 */
  int ntrial_first, ntrial;
  uint64_t seed;
  uint32_t sys_id;
  int smem_fw;                /* framework staged in shared memory by the engine */
  /* flexible linear chain (rgpu_system_desc), grown from atom 0 */
  int flexible;
  int pad_flex;
  double bond, bend_k, bend_theta0, bend_sigma;   /* bend_sigma = 1 / sqrt(beta bend_k) */
  double torsion[4], torsion_min;                 /* torsion_min: minimum of the torsion energy over phi */
  int chain_scheme;           /* rgpu_system_desc.chain_scheme: 0 the reference's bonded trials, 1 independent draws */
  int ntors;                  /* torsion candidates per trial (chain_scheme 0) */
  /* energy grids (rgpu_system_set_grids): the engine takes the host VDW
   * energy of molecule atom a from grid[a] instead of the pair sums */
  int use_grid;
  int use_coul_grid;          /* host real-space charge energy from coul_grid (x the bead charge) */
  RgpuGridGeom grid_geom;
  const float *grid[RGPU_MAX_ATOMS];
  RgpuGridGeom coul_geom;
  const float *coul_grid;     /* Coulomb grid of a unit probe charge (rgpu_system_set_coulomb_grid) */
  /* device pointers */
  const double4 *fw64;        /* [nfw] x, y, z, q (sorted by type) */
  const int4 *fw32;           /* [ntile*RGPU_TILE] tiled: fixed-point x, y, z (low 2 bits of z = segment), float bits of q */
  const TileRec *tiles;       /* [ntile] */
  int ntile;
  int pad_tile;
  const char4 *kvec;          /* [nk] */
  const double *kfactor;      /* [nk] */
  const double2 *sk_fw;       /* [nk] */
  double2 *sk_ads;            /* [nk] */
  double *ads_xyz;            /* [maxmol*natom*3] authoritative positions */
  int *nmol;                  /* [1] */
  double *energy;             /* [RGPU_NE] running totals (inside the RgpuState block) */
  unsigned long long *step;   /* [4], see RgpuState.step */
  long long *counters;        /* [RGPU_NCNT] */
  double *sums;               /* [RGPU_NSUM] */
  int *status;                /* [1] */
} RgpuSys;

#endif
