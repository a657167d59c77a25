/* raspa_gpu.h — C ABI of the B200 GCMC energy path (libraspa_gpu.so).
 *
 * The reference (RASPA2) evaluates every Monte Carlo energy through a small
 * set of C routines over process-global state; its host MC loop
 * (src/mc_moves.c, src/cbmc.c) calls them once per trial position or move.
 * This library exports the same operations over an explicit system handle,
 * with plain pointers and sizes, so that a patched copy of those routines can
 * forward to the GPU, plus batched entry points that
 * evaluate a whole CBMC trial set per call and a persistent engine that runs
 * many independent systems entirely on the device.
 *
 * Units: lengths in Angstrom, charges in e, energies in the reference's
 * internal unit (amu A^2 / ps^2; src/constants.c:147). Positions are
 * Cartesian, row-major [n][3] doubles. All calls are synchronous on the
 * library's stream unless stated; none of them exits the process: every
 * function returns 0 (RGPU_SUCCESS) or a negative error code
 * (rgpu_error_string() describes it).
 */
#ifndef RASPA_GPU_H
#define RASPA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RGPU_SUCCESS 0
#define RGPU_E_INVALID -1      /* bad argument or size beyond a compiled limit */
#define RGPU_E_CUDA -2         /* a CUDA runtime call failed (see rgpu_error_string) */
#define RGPU_E_NODEVICE -3     /* no CUDA device */
#define RGPU_E_CAPACITY -4     /* molecule capacity of the system exceeded */
#define RGPU_E_IO -5           /* a file could not be opened, read or written, or is not a grid file */

/* precision of a call */
#define RGPU_FP64 0            /* FP64 throughout (the reference's REAL) */
#define RGPU_MIXED 1           /* FP32 pair terms / FP64 sums and S(k) */
#define RGPU_MIXED_CC64 2      /* as RGPU_MIXED, with each pair's distance, cut-off test and
                                * real-space charge-charge term, and the Fourier phases and
                                * dS(k), in FP64; LJ terms stay FP32 (rgpu_engine_create
                                * only; rigid molecules without energy grids) */

typedef struct rgpu_system rgpu_system;
typedef struct rgpu_engine rgpu_engine;

/* Description of one simulation box (rigid framework + one rigid adsorbate
 * component). Replaces what the reference reads into Framework[],
 * Components[], PseudoAtoms and the Ewald globals (src/input.c ReadInputFile,
 * src/ewald.c:200-261 InitializeEwald, :532-599 SetupKVectors). */
typedef struct {
  double box[3];              /* orthorhombic box lengths; each >= 2 * cutoff (see cell_matrix) */
  double cutoff;              /* VDW and real-space charge cut-off */
  double beta;                /* 1 / (k_B T), inverse internal energy units */
  double coulomb;             /* COULOMBIC_CONVERSION_FACTOR (src/constants.c:162) */
  double overlap;             /* EnergyOverlapCriteria (src/input.c:367) */
  int nfw;                    /* framework atoms */
  const double *fw_xyz;       /* [nfw][3] */
  const int *fw_type;         /* [nfw] pseudo-atom type (index into the LJ table) */
  const double *fw_q;         /* [nfw] charge */
  int ntypes;                 /* LJ table dimension */
  const double *eps;          /* [ntypes*ntypes] epsilon (internal units), mixed */
  const double *sig2;         /* [ntypes*ntypes] sigma^2 */
  const double *shift;        /* [ntypes*ntypes] U(cutoff) (0 for truncated) */
  int natom;                  /* atoms per adsorbate molecule (<= 8) */
  const int *mol_type;        /* [natom] */
  const double *mol_q;        /* [natom] */
  const double *mol_ref;      /* [natom][3] rigid reference geometry */
  int start_bead;             /* CBMC starting bead */
  int ewald;                  /* 1: Ewald summation (charges), 0: no charges */
  double alpha;               /* Ewald screening parameter */
  int kmax[3];                /* wave vectors per axis */
  int maxmol;                 /* molecule capacity */
  /* MC move parameters (used by the engine) */
  double move_cum[6];         /* cumulative probabilities: translate, rotate, insert, delete,
                                 reinsert, Widom test insertion */
  double max_translation;     /* Angstrom */
  double max_rotation;        /* radian */
  double fugacity_beta_v;     /* beta * fugacity * volume (ideal-gas Rosenbluth weight 1) */
  int ntrial_first;           /* NumberOfTrialPositionsForTheFirstBead (<= 16) */
  int ntrial;                 /* NumberOfTrialPositions (<= 16) */
  uint64_t seed;              /* random stream seed */
  uint32_t stream_id;         /* random stream id of this system */
  /* Flexible linear chain (e.g. united-atom alkanes): atoms 0..natom-1 in
   * chain order, grown from atom 0 (start_bead must be 0), uncharged. Fixed
   * bond length, one harmonic bend 0.5 bend_k (theta - bend_theta0)^2 per
   * atom triple, one TraPPE torsion t0 + t1 (1 + cos phi) + t2 (1 - cos 2 phi)
   * + t3 (1 + cos 3 phi) per quadruple (src/internal_energy.c TRAPPE_DIHEDRAL,
   * HARMONIC_BEND), LJ between atoms four or more bonds apart. Energies in
   * internal units, angles in radians. flexible = 0: rigid molecule
   * (mol_ref is its geometry). */
  int flexible;
  double bond;
  double bend_k, bend_theta0;
  double torsion[4];
  /* Bonded part of a chain's CBMC trials. chain_scheme 0 (the reference's
   * GenerateTrialOrientationsMCScheme, src/cbmc.c:1580-2480): one bend angle
   * per growth step, drawn from sin(theta) exp(-beta U_bend) and shared by
   * the step's trials (a retrace keeps the old angle); per trial `ntors`
   * uniform rotations about the previous bond, one chosen by its torsion
   * Boltzmann factor; the weight carries the chosen trial's torsion
   * Rosenbluth factor, averaged, as the reference averages it, over the
   * first ntrial candidates (src/cbmc.c:548, :2401, :2793). ntors = 0 means
   * the reference's default NumberOfTrialPositionsTorsion, 100 (at most
   * 128). chain_scheme 1: each trial draws its own bend angle and dihedral
   * from their Boltzmann distributions (no torsion factor in the weight). */
  int chain_scheme;
  int ntors;
  /* Triclinic box (BoundaryCondition TRICLINIC): the box matrix, row-major,
   * whose columns are the cell vectors a, b, c, upper triangular as the
   * reference builds Box (a along x, b in the xy plane; src/framework.c:
   * 2025-2040). All zero: the orthorhombic box of box[3]. Every
   * perpendicular width must be >= 2 * cutoff. Distances use the
   * reference's triclinic minimum image (fractional coordinates wrapped to
   * the nearest integer, src/potentials.h:246-262), wave vectors 2 pi H^-T n
   * (src/ewald.c:560-595). Energy grids span the enclosing box of the unit
   * cell and their lookups wrap a point into the unit cell through its
   * fractional coordinates (src/grids.c:336-360, :1004-1021); the unit cell
   * is the box's with the cell lengths passed to the grid calls. */
  double cell_matrix[9];
} rgpu_system_desc;

const char *rgpu_error_string(int code);
int rgpu_device_count(void);

/* ---- system lifetime and adsorbate state -------------------------------- */
int rgpu_system_create(rgpu_system **out, const rgpu_system_desc *desc);
int rgpu_system_destroy(rgpu_system *sys);
/* Replaces the adsorbate configuration (nmol molecules, [nmol][natom][3]) and
 * recomputes the stored structure factors; the state the reference builds
 * with InsertAdsorbateMolecule (src/molecule.c:3075) and
 * PrecomputeTotalEwaldContributions (src/ewald.c:1289). */
int rgpu_set_adsorbates(rgpu_system *sys, int nmol, const double *xyz);
int rgpu_get_adsorbates(rgpu_system *sys, int *nmol, double *xyz, int capacity);
/* Moves molecule m to xyz ([natom][3]) after an accepted displacement
 * (src/mc_moves.c:1743-1748); appends / removes a molecule (the last one
 * takes the freed slot, src/molecule.c:3193 RemoveAdsorbateMolecule). These
 * update positions only; S(k) follows through rgpu_ewald_accept. */
int rgpu_update_molecule(rgpu_system *sys, int m, const double *xyz);
int rgpu_insert_molecule(rgpu_system *sys, const double *xyz);
int rgpu_remove_molecule(rgpu_system *sys, int m);

/* ---- energies (the reference's per-call routines) ------------------------ */
/* Energies of `n` bead positions in one call:
 *   out[4*i+0] host VDW      CalculateFrameworkVDWEnergyAtPosition   src/framework_energy.c:60
 *   out[4*i+1] host charge   CalculateFrameworkChargeEnergyAtPosition src/framework_energy.c:176
 *   out[4*i+2] adsorbate VDW CalculateInterVDWEnergyAdsorbateAtPosition src/inter_energy.c:321
 *   out[4*i+3] adsorbate q   CalculateInterChargeEnergyAdsorbateAtPosition src/inter_energy.c:393
 * xyz[n][3]; atom[i] = index of the bead in the molecule (type and charge);
 * exclude[i] = adsorbate molecule left out (-1 for none). Batched form of the
 * trial loops of HandleFirstBead (src/cbmc.c:644-743) and
 * ComputeExternalEnergies (src/cbmc.c:1179-1476). n <= 64 per call. */
int rgpu_bead_energies(rgpu_system *sys, int precision, int n, const double *xyz, const int *atom,
                       const int *exclude, double *out);

/* Energy differences of molecule m moved to new_xyz ([natom][3]):
 *   out = {dU host VDW, dU host charge, dU adsorbate VDW, dU adsorbate charge}
 * CalculateFrameworkAdsorbateVDWEnergyDifference (src/framework_energy.c:4870),
 * CalculateFrameworkAdsorbateChargeChargeEnergyDifference (:5412),
 * CalculateInterVDWEnergyDifferenceAdsorbate (src/inter_energy.c:3071),
 * CalculateInterChargeChargeEnergyDifferenceAdsorbate (:3652).
 * *overlap = 1 when a new-position pair energy reaches the overlap criterion
 * (the routines' `return OVERLAP=TRUE`). */
int rgpu_move_energy_difference(rgpu_system *sys, int precision, int m, const double *new_xyz, double *out,
                                int *overlap);

/* Ewald Fourier difference, CalculateEwaldFourierAdsorbate(New, Old, mol,
 * store) (src/ewald.c:6859): old_mol >= 0 removes that molecule's sites,
 * new_xyz != NULL adds a molecule at new_xyz. out = {dU adsorbate-adsorbate
 * Fourier, dU host-adsorbate Fourier, net charge change}. The candidate
 * S(k) is kept on the device until rgpu_ewald_accept. */
int rgpu_ewald_fourier_difference(rgpu_system *sys, int precision, int old_mol, const double *new_xyz,
                                  double *out);
/* AcceptEwaldAdsorbateMove (src/ewald.c:11732): the candidate becomes S(k). */
int rgpu_ewald_accept(rgpu_system *sys);

/* Total energies of the current configuration recomputed from scratch
 * (CalculateEnergy, src/integration.c:250): out = {host VDW, adsorbate VDW,
 * host real, adsorbate real, host Fourier, adsorbate Fourier}. FP64. */
int rgpu_total_energy(rgpu_system *sys, double *out);

/* Intramolecular energy (bends, torsions, LJ of atoms four or more bonds
 * apart) of all molecules of a flexible-chain system, recomputed from the
 * current positions; 0 for rigid molecules. The engine's running value is
 * energy8[6] of rgpu_system_state. */
int rgpu_intra_energy(rgpu_system *sys, double *out);

/* ---- energy grids (src/grids.c) ----------------------------------------- */
/* MakeGrid (src/grids.c:431-690) for pseudo-atom `type`: (n+1)^3 points
 * i*size/n + shift per axis, 8 FP32 values per point (value, 3 first, 3 mixed
 * second, 1 third derivative, scaled to the unit cell of the grid), stored
 * point-major: grid[((i*(ny+1) + j)*(nz+1) + k)*8 + m], so that a lookup
 * reads each corner's 8 values as two 16-byte loads. The reference's grid
 * file holds the same values plane by plane (src/grids.c:734-738): plane m
 * is grid[...*8 + m]. d_grid is 16-byte aligned device memory of
 * (nx+1)(ny+1)(nz+1)*8 floats. */
int rgpu_grid_build(rgpu_system *sys, int type, const int npts[3], const double size[3],
                    const double shift[3], float *d_grid);
/* The Coulomb grid (MakeGrid's electrostatic part, src/grids.c:586-690,
 * with CalculateDerivativesAtPositionReal, src/framework_hessian.c:111-180):
 * the real-space Ewald energy K q_fw erfc(alpha r)/r of a unit probe charge
 * with the framework, with the same 8 values per point and the same layout
 * as rgpu_grid_build; a point within 1 A of a framework atom, or above the
 * overlap criterion, is capped as the reference caps it. Needs Ewald. The
 * reference makes the point counts odd (int(size/spacing), +1 if even). */
int rgpu_grid_build_coulomb(rgpu_system *sys, const int npts[3], const double size[3], const double shift[3],
                            float *d_grid);
/* InterpolateVDWGrid (src/grids.c:979-1077) at n points (host arrays),
 * reading the device grid; cell = the unit-cell lengths the grid spans.
 * The same lookup serves a Coulomb grid (InterpolateCoulombGrid,
 * src/grids.c:1200-1295, before the multiplication by the bead charge): its
 * capped points hold 2e7, below the VDW lookup's 1e10 corner test. */
int rgpu_grid_interpolate(const float *d_grid, const int npts[3], const double size[3], const double shift[3],
                          const double cell[3], int n, const double *xyz, double *out);

/* ---- grid files --------------------------------------------------------- */
/* The reference's grid files: WriteVDWGrid / ReadVDWGrid (src/grids.c:692-813)
 * and WriteCoulombGrid / ReadCoulombGrid (:815-977). A file is the header
 * below, in the fields' native binary form and this order (REAL = double,
 * INT_VECTOR3 = 3 ints, VECTOR = 3 doubles; 128 bytes, 136 with the Coulomb
 * file's Ewald precision), then the 8 values of every grid point as 8 planes
 * of (npts[0]+1)(npts[1]+1)(npts[2]+1) floats, [m][i][j][k]. On the device a
 * grid is point-major ([i][j][k][m], the layout of rgpu_grid_build); the
 * calls below transpose between the two on the GPU. */
typedef struct rgpu_grid_file_header {
  double spacing;       /* SpacingVDWGrid / SpacingCoulombGrid */
  int npts[3];          /* NumberOfVDWGridPoints / NumberOfCoulombGridPoints */
  double size[3];       /* SizeGrid */
  double shift[3];      /* ShiftGrid */
  double delta[3];      /* DeltaVDWGrid / DeltaCoulombGrid */
  double unit_cell[3];  /* UnitCellSize */
  int unit_cells[3];    /* NumberOfUnitCells */
  double ewald_precision; /* EwaldPrecision: Coulomb files only */
} rgpu_grid_file_header;
/* Reads the header of the grid file at `path` (coulomb = 1 for a Coulomb
 * grid file) and checks that the file holds exactly the grid it announces;
 * RGPU_E_IO otherwise. */
int rgpu_grid_read_file_header(const char *path, int coulomb, rgpu_grid_file_header *hdr);
/* Reads the grid file into d_grid (device, 16-byte aligned, capacity in
 * floats >= 8 (npts+1)^3) in the device layout, and its header into hdr.
 * The caller checks hdr->unit_cell (and, for a Coulomb grid,
 * hdr->unit_cells) against the system, as ReadVDWGrid and ReadCoulombGrid
 * do (src/grids.c:787-792, :936-949). Uses a temporary device buffer of the
 * grid's size; returns when the grid is in place. */
int rgpu_grid_read_file(const char *path, int coulomb, rgpu_grid_file_header *hdr, float *d_grid, size_t capacity);
/* Writes the device grid d_grid (npts from hdr) with header hdr to `path`
 * in the reference's format, creating missing parent directories (mode
 * 0700, as WriteVDWGrid's mkdir calls). */
int rgpu_grid_write_file(const char *path, int coulomb, const rgpu_grid_file_header *hdr, const float *d_grid);
/* The path the reference gives a grid file, written into buf (size n):
 * <raspa_dir>/share/raspa/grids/<forcefield>/<framework>/<spacing %lf>/ then
 * <framework>_<pseudo_atom>_<shifted|truncated>.grid for a VDW grid
 * (src/grids.c:716-723), or, when pseudo_atom is NULL, the Coulomb grid's
 * <ncx>x<ncy>x<ncz>/<framework>_Electrostatics_<method>.grid with method
 * "Ewald" (:841-853; unit_cells required then). RGPU_E_INVALID when buf is
 * too small. */
int rgpu_grid_file_path(char *buf, size_t n, const char *raspa_dir, const char *forcefield, const char *framework,
                        double spacing, const char *pseudo_atom, int shifted, const int unit_cells[3]);

/* ---- grid lookup without device allocation ------------------------------ */
/* No counterpart in the reference. Same result as rgpu_grid_interpolate for
 * n <= RGPU_NOALLOC_MAX_POINTS points, but the call makes no device
 * allocation: positions and results pass through a file-scope device array of
 * 256 KB (one per device) instead of buffers allocated per call. The first
 * call on each device looks up that array's address (cudaGetSymbolAddress)
 * with the device current and keeps it, so make the first call before any
 * stream capture. The kept address belongs to the device's current context:
 * it does not survive cudaDeviceReset, so do not call this after a reset in
 * the same process. n above RGPU_NOALLOC_MAX_POINTS returns RGPU_E_INVALID.
 * Calls that overlap on one device (several host threads) share the array
 * and race: serialise them. Runs on the legacy default stream, synchronises
 * that stream and returns when the results are in `out`. */
#define RGPU_NOALLOC_MAX_POINTS 8192
int rgpu_grid_interpolate_noalloc(const float *d_grid, const int npts[3], const double size[3],
                                  const double shift[3], const double cell[3], int n, const double *xyz,
                                  double *out);

/* Uses energy grids in the engine: the host VDW energy of molecule atom a
 * becomes the tricubic lookup in d_grids[a] (a grid of rgpu_grid_build for
 * that atom's pseudo-atom type; atoms of one type can share a grid) instead
 * of the pair sum over the framework, as the reference does with
 * UseTabularGrid (src/grids.c:979, called from src/framework_energy.c).
 * npts/size/shift/cell as rgpu_grid_interpolate; a charged molecule needs a
 * Coulomb grid (rgpu_system_set_coulomb_grid) set first. d_grids = NULL switches the grids off (and sets the
 * FULL framework model below). Takes effect for engines created afterwards;
 * the per-call energies (rgpu_bead_energies, rgpu_move_energy_difference,
 * rgpu_total_energy) keep the direct pair sums unless the framework model is
 * RGPU_FRAMEWORK_GRID. */
int rgpu_system_set_grids(rgpu_system *sys, const float *const *d_grids, const int npts[3], const double size[3],
                          const double shift[3], const double cell[3]);
/* The Coulomb grid of the engine (a grid of rgpu_grid_build_coulomb): the
 * host real-space charge energy of a bead becomes its charge times the
 * lookup, as the reference's grid framework model does
 * (src/framework_energy.c:195-198, :5437-5438); the Fourier part stays
 * ΔS(k). Set it before rgpu_system_set_grids when the molecule is charged.
 * d_grid = NULL removes it (refused while VDW grids of a charged molecule
 * are on). */
int rgpu_system_set_coulomb_grid(rgpu_system *sys, const float *d_grid, const int npts[3], const double size[3],
                                 const double shift[3], const double cell[3]);

/* ---- framework model of the per-call energies --------------------------- */
/* Framework[].FrameworkModel (src/framework.h) for the per-call routines:
 * RGPU_FRAMEWORK_FULL (the default) sums the framework pairs;
 * RGPU_FRAMEWORK_GRID takes the framework terms from the grids set with
 * rgpu_system_set_grids / rgpu_system_set_coulomb_grid, as the reference
 * does when the model is GRID: the framework VDW energy of a bead of
 * molecule atom a is the lookup in atom a's grid
 * (CalculateFrameworkVDWEnergyAtPosition, src/framework_energy.c:73-77), its
 * real-space charge energy the bead charge times the Coulomb-grid lookup
 * (CalculateFrameworkChargeEnergyAtPosition, :195-198), and the same in the
 * move differences (:4893-4894, :5437-5438) and the totals (:2707, :2920).
 * rgpu_bead_energies, rgpu_move_energy_difference and rgpu_total_energy
 * follow the model; the engine uses the grids whenever they are set. A grid
 * value raises no overlap flag in rgpu_move_energy_difference (the
 * reference's grid branch sets none; a capped lookup returns 1e8, which the
 * acceptance rule rejects). GRID without grids set, or an unknown model,
 * returns RGPU_E_INVALID. */
#define RGPU_FRAMEWORK_FULL 0
#define RGPU_FRAMEWORK_GRID 1
int rgpu_system_set_framework_model(rgpu_system *sys, int model);

/* ---- persistent batched engine ------------------------------------------ */
/* Groups systems for one persistent launch; each system is advanced by one
 * thread-block cluster of `cluster` CTAs (1 to 8; 0 chooses from the
 * number of systems and SMs) that split its framework between them.
 * `threads` = CTA size, a multiple of 32 in 64..1024 (RGPU_MIXED,
 * RGPU_MIXED_CC64) or 64..512 (RGPU_FP64). */
int rgpu_engine_create(rgpu_engine **out, rgpu_system *const *systems, int n, int precision, int threads,
                       int cluster);
/* As rgpu_engine_create, with the shared memory and registers of each CTA
 * sized so that `ctas_per_sm` CTAs (1..4) can share one SM: CTAs of
 * different systems then interleave on an SM and fill each other's barrier
 * waits. Framework and wave vectors that no longer fit are read from global
 * memory (L2). No counterpart in the reference. */
int rgpu_engine_create_ex(rgpu_engine **out, rgpu_system *const *systems, int n, int precision, int threads,
                          int cluster, int ctas_per_sm);
/* CTAs per system of an engine. */
int rgpu_engine_cluster(rgpu_engine *eng);
/* Runs the systems second[0..nsecond) (indices into the engine's systems)
 * in a second launch with clusters of `cluster_b` CTAs (1 to 8), side
 * by side with the launch of the others on a stream of the engine's own;
 * rgpu_engine_run's stream waits for both. One cluster size per launch, so
 * this is how the costliest systems get more CTAs, on SMs a single launch
 * would leave idle. nsecond = 0 returns to one launch. Synchronises the
 * device. No counterpart in the reference. */
int rgpu_engine_set_split(rgpu_engine *eng, const int *second, int nsecond, int cluster_b);
int rgpu_engine_destroy(rgpu_engine *eng);
/* Advances every system by `nsteps` MC moves (asynchronous on `stream`, a
 * cudaStream_t or NULL for the library stream). RGPU_E_INVALID if a system
 * was given energy grids after an engine without the flexible-chain/grid
 * build was created over it. */
int rgpu_engine_run(rgpu_engine *eng, long long nsteps, void *stream);
int rgpu_engine_sync(rgpu_engine *eng);
/* With `on` != 0, rgpu_engine_run replays a CUDA graph of the launch
 * (captured on the first run, and again whenever nsteps changes) instead
 * of launching the kernel directly. */
int rgpu_engine_use_graph(rgpu_engine *eng, int on);
/* Replaces system i (creation order) of the engine by `sys` in place, for a
 * request loop that admits jobs into the slots of finished ones: one
 * asynchronous copy on `stream` (a cudaStream_t, NULL for the library
 * stream), ordered after the launches already queued there, with no
 * allocation, no device synchronisation and a captured graph left valid.
 * The new system must fit the engine's launch layout (molecule capacity,
 * Ewald phase tables, kernel build) and the engine must have no batched
 * staging buffer; otherwise RGPU_E_INVALID and the caller builds a new
 * engine. A system at its step limit takes no step in a launch, so a
 * finished job can stay in its slot until it is replaced; the replaced
 * system may be destroyed once `stream` has passed the copy. No
 * counterpart in the reference. */
int rgpu_engine_replace_system(rgpu_engine *eng, int i, rgpu_system *sys, void *stream);
/* Running energies (8 doubles, first six as rgpu_total_energy), counters
 * (20: attempts[4] and accepted[4] of translation, rotation, insertion,
 * deletion; counted moves, overlaps, pairs visited, pairs in cut-off,
 * charged pairs in cut-off, k x site products, k sums, engine clock cycles,
 * of which in pair evaluations, in Ewald sums; reinsertions attempted,
 * accepted), molecule count, status word (0 = fine) and next step index. */
int rgpu_system_state(rgpu_system *sys, double *energy8, long long *counters20, int *nmol, int *status,
                      unsigned long long *step);
/* Resets the running energies to `energy8` (e.g. after rgpu_total_energy). */
int rgpu_system_set_energy(rgpu_system *sys, const double *energy8);
/* Step window of a system in the engine: rgpu_engine_run stops advancing it
 * at step `end_step` (exclusive; 0 = no limit), and steps from `avg_start`
 * on enter the ensemble sums. The reference samples its averages once per
 * cycle (src/monte_carlo.c:580, src/statistics.c:1112); the engine samples
 * once per MC step. The limits take effect from the next engine launch;
 * call this between launches of an engine that holds the system (it does
 * not wait for other work on the device). */
int rgpu_system_set_limits(rgpu_system *sys, unsigned long long end_step, unsigned long long avg_start);
/* Ensemble sums: {steps sampled, sum N, sum N^2, sum U, sum U*N, sum U^2,
 * sum of Widom Rosenbluth weights, Widom samples}, U = the six running
 * energy terms added, N = molecules. Loading <N>, energy <U> and the
 * enthalpy of adsorption (<UN> - <U><N>) / (<N^2> - <N>^2) - k_B T
 * (src/statistics.c:4077-4079) follow from the first six; the average Widom
 * weight <W> (src/mc_moves.c:7844-8030; an overlapping test insertion counts
 * with W = 0) gives the excess chemical potential -k_B T ln <W> and the
 * Henry coefficient beta <W> per unit volume. Widom samples are taken at
 * every Widom step, whatever the step window. */
int rgpu_system_averages(rgpu_system *sys, double *sums8);
int rgpu_system_reset_averages(rgpu_system *sys);

/* ---- batched state transfer of an engine's systems ------------------------ */
/* No counterpart in the reference (its state is host memory). The
 * per-system calls below cost a synchronisation each; these move all
 * systems of an engine through one pinned staging buffer, with one copy and
 * one synchronisation per call.
 *
 * rgpu_engine_get_state: for system i of the engine (creation order),
 * energy8[8i..], counters20[20i..], nmol[i], status[i], step[i] as
 * rgpu_system_state, and its positions into xyz[i] (room for maxmol * natom
 * * 3 doubles; xyz or xyz[i] may be NULL) as rgpu_get_adsorbates. Any output
 * pointer may be NULL.
 *
 * rgpu_engine_set_adsorbates: as rgpu_set_adsorbates(sys_i, nmol[i],
 * xyz[i]) for every system: positions, molecule count, the per-call
 * records and S_ads(k) from the new positions; running energies untouched.
 *
 * Both wait for the device first (no engine launch may be in flight). */
int rgpu_engine_get_state(rgpu_engine *eng, double *energy8, long long *counters20, int *nmol, int *status,
                          unsigned long long *step, double *const *xyz);
int rgpu_engine_set_adsorbates(rgpu_engine *eng, const int *nmol, const double *const *xyz);
/* Bytes each of those calls copies between host and device (the whole
 * staging buffer: every system's state block and room for maxmol molecules). */
int rgpu_engine_staging_bytes(rgpu_engine *eng, size_t *bytes);

/* ---- checkpoints (binary crash files) ------------------------------------ */
/* The counterpart of the binary crash file that ContinueAfterCrash writes
 * and reads (WriteBinaryRestartFiles, src/output.c:7903;
 * ReadBinaryRestartFiles, src/input.c:9378): a system's whole mutable state
 * as one host buffer. It holds the molecule positions (FP64), the stored
 * adsorbate structure factor S_ads(k) as updated move by move (FP64), the
 * running energies, counters, ensemble sums, step window and status word.
 * The random stream is keyed by step, and the step is saved, so a system
 * created from the same descriptor (same seed and stream id) and restored
 * from a checkpoint continues the saved trajectory move for move. Restoring
 * into a system of another temperature, pressure, move mix or stream is
 * allowed; another box, framework, force field, molecule or Ewald set-up is
 * refused (RGPU_E_INVALID). Energy grids are part of the descriptor, not of
 * the state: set them on the restoring system. The buffer is host memory of
 * rgpu_system_checkpoint_size bytes (it grows with the molecule count). */
int rgpu_system_checkpoint_size(rgpu_system *sys, size_t *bytes);
int rgpu_system_checkpoint(rgpu_system *sys, void *buf, size_t bytes);
int rgpu_system_restore(rgpu_system *sys, const void *buf, size_t bytes);

/* ---- measurement -------------------------------------------------------- */
/* FP32 FMA throughput of the current device in TFLOP/s (FMA = 2 FLOP), the
 * roofline denominator of the pair kernels. No counterpart in the reference. */
int rgpu_fp32_peak_probe(double *tflops, double *seconds);

#ifdef __cplusplus
}
#endif
#endif
