/* raspa_gpu_bridge.c — RASPA2's per-call energy routines on libraspa_gpu.
 *
 * Linked into the reference program with the linker's --wrap option (see
 * oracle/Makefile, target simulate_gpu): every call that src/cbmc.c and
 * src/mc_moves.c make to the routines below lands in the __wrap_ function
 * here, which evaluates it on the GPU through the C ABI of include/raspa_gpu.h
 * and writes the reference's own outputs (return values and the U*Delta /
 * OVERLAP globals). The reference's sources are not changed; they are only
 * compiled against (their headers declare the globals read here).
 *
 *   CalculateFrameworkVDWEnergyAtPosition           src/framework_energy.c:60
 *   CalculateFrameworkChargeEnergyAtPosition        src/framework_energy.c:176
 *   CalculateInterVDWEnergyAdsorbateAtPosition      src/inter_energy.c:321
 *   CalculateInterChargeEnergyAdsorbateAtPosition   src/inter_energy.c:393
 *   CalculateFrameworkAdsorbateVDWEnergyDifference  src/framework_energy.c:4870
 *   CalculateFrameworkAdsorbateChargeChargeEnergyDifference  src/framework_energy.c:5412
 *   CalculateInterVDWEnergyDifferenceAdsorbate      src/inter_energy.c:3071
 *   CalculateInterChargeChargeEnergyDifferenceAdsorbate      src/inter_energy.c:3652
 *   CalculateEwaldFourierAdsorbate                  src/ewald.c:6859
 *   AcceptEwaldAdsorbateMove                        src/ewald.c:11732
 *   MakeGrid                                        src/grids.c:431
 *
 * The GPU system is built from the reference's globals on the first call
 * (the input has been read and Ewald set up by then). The adsorbate
 * positions on the device follow Adsorbates[][]: before each call the
 * bridge compares them with its copy and uploads them when they changed (an
 * accepted move, an insertion or a removal), which also recomputes the
 * stored S(k) from the positions.
 *
 * The four energies of a point are computed in one device call and served
 * to the four at-position routines that the reference calls one after the
 * other for the same point (src/cbmc.c:680-697); the four move differences
 * likewise (src/mc_moves.c:1598-1623).
 *
 * Supported: one system, one adsorbate component (rigid or single-bead; a
 * flexible chain's external energies as well), one rigid framework, an
 * orthorhombic or triclinic box without replicas or cell lists, Lennard-Jones (or zero)
 * potentials, charges by the Ewald method with one cut-off, no CFCMC
 * scaling. With the GRID framework model (UseTabularGrid) the grid files
 * the reference read at start-up (the VDW grid of every adsorbate
 * pseudo-atom, and the Coulomb grid for a charged adsorbate) are read once
 * more, by the library's reader, into device memory, and the per-call
 * routines take the framework terms from them
 * (rgpu_system_set_framework_model). Anything else stops the
 * program with a message, as the reference's own fatal paths do (fprintf,
 * exit); no routine falls back to the CPU.
 *
 * Environment: RASPA_GPU_PRECISION=mixed selects the mixed-precision path
 * (default FP64); RASPA_GPU_BRIDGE_STATS=1 prints the number of device
 * calls per routine at exit.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "constants.h"
#include "simulation.h"
#include "molecule.h"
#include "framework.h"
#include "potentials.h"
#include "ewald.h"
#include "cbmc.h"
#include "mc_moves.h"

#include "grids.h"
#include "output.h"

#include <cuda_runtime_api.h>

#include "raspa_gpu.h"

#define BRIDGE_MAXMOL 4096
#define BRIDGE_MAXTYPES 4096

static rgpu_system *g_sys;
static int g_system = -1, g_comp = -1, g_natom = 0, g_prec = RGPU_FP64;
static int g_atom_of_type[BRIDGE_MAXTYPES];
static double *g_mirror;          /* adsorbate positions on the device, [nmol][natom][3] */
static double *g_scratch;
static int g_mirror_n = -1;
static int g_pending_store = -1;  /* store index of the candidate S(k) on the device */
static long long g_calls[4];      /* point energies, differences, Ewald, uploads */

static void bridge_fail(const char *what, int rc)
{
  fprintf(stderr, "raspa_gpu_bridge: %s%s%s\n", what, rc ? ": " : "", rc ? rgpu_error_string(rc) : "");
  exit(2);
}

static void print_stats(void)
{
  fprintf(stderr, "raspa_gpu_bridge: device calls: point energies %lld, move differences %lld, Ewald %lld, "
                  "configuration uploads %lld\n",
          g_calls[0], g_calls[1], g_calls[2], g_calls[3]);
}

/* a grid file of the reference (the one ReadVDWGrid / ReadCoulombGrid read
 * before the first call) into a new device buffer, through the library's
 * reader; the header must match the grid the reference holds */
static float *bridge_read_grid(const char *pseudo_atom, int coulomb, int s, rgpu_grid_file_header *h)
{
  char path[4096];
  const int nc[3] = {NumberOfUnitCells[s].x, NumberOfUnitCells[s].y, NumberOfUnitCells[s].z};
  int rc = rgpu_grid_file_path(path, sizeof path, RASPA_DIRECTORY, ForceField, Framework[s].Name[0],
                               coulomb ? SpacingCoulombGrid : SpacingVDWGrid, coulomb ? NULL : pseudo_atom,
                               ShiftPotentials, nc);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_file_path", rc);
  rc = rgpu_grid_read_file_header(path, coulomb, h);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_read_file_header", rc);
  if (fabs(h->unit_cell[0] - UnitCellSize[s].x) > 1e-8 || fabs(h->unit_cell[1] - UnitCellSize[s].y) > 1e-8 ||
      fabs(h->unit_cell[2] - UnitCellSize[s].z) > 1e-8)
    bridge_fail("grid file: unit-cell size does not match", 0);
  if (!coulomb && (h->npts[0] != NumberOfVDWGridPoints.x || h->npts[1] != NumberOfVDWGridPoints.y ||
                   h->npts[2] != NumberOfVDWGridPoints.z))
    bridge_fail("grid file: number of grid points does not match the reference's grid", 0);
  const size_t n = (size_t)8 * (h->npts[0] + 1) * (h->npts[1] + 1) * (h->npts[2] + 1);
  float *d = NULL;
  if (cudaMalloc((void **)&d, sizeof(float) * n) != cudaSuccess) bridge_fail("cudaMalloc of a grid", 0);
  rc = rgpu_grid_read_file(path, coulomb, h, d, n);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_read_file", rc);
  return d;
}

/* the GRID framework model (src/framework_energy.c:73-77, :195-198): every
 * adsorbate pseudo-atom needs its VDW grid, a charged adsorbate the Coulomb
 * grid; the device grids live until the program exits */
static void bridge_grids(const COMPONENT *C, int s)
{
  const float *ptr[64];
  float *by_type[BRIDGE_MAXTYPES];
  memset(by_type, 0, sizeof by_type);
  rgpu_grid_file_header h;
  int charged = 0;
  for (int a = 0; a < C->NumberOfAtoms; a++) {
    const int t = C->Type[a];
    if (!VDWGrid || !VDWGrid[t]) bridge_fail("the GRID framework model needs a VDW grid of every adsorbate atom", 0);
    if (!by_type[t]) by_type[t] = bridge_read_grid(PseudoAtoms[t].Name, 0, s, &h);
    ptr[a] = by_type[t];
    charged |= C->Charge[a] != 0.0;
  }
  int rc;
  if (charged && ChargeMethod == EWALD) {
    if (!CoulombGrid) bridge_fail("the GRID framework model of a charged adsorbate needs the Coulomb grid", 0);
    rgpu_grid_file_header hc;
    float *dc = bridge_read_grid(NULL, 1, s, &hc);
    rc = rgpu_system_set_coulomb_grid(g_sys, dc, hc.npts, hc.size, hc.shift, hc.unit_cell);
    if (rc != RGPU_SUCCESS) bridge_fail("rgpu_system_set_coulomb_grid", rc);
  }
  rc = rgpu_system_set_grids(g_sys, ptr, h.npts, h.size, h.shift, h.unit_cell);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_system_set_grids", rc);
  rc = rgpu_system_set_framework_model(g_sys, RGPU_FRAMEWORK_GRID);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_system_set_framework_model", rc);
}

/* the GPU system from the reference's globals (src/input.c, src/ewald.c:200-261) */
static void bridge_init(void)
{
  const int s = CurrentSystem;
  if (g_sys) {
    if (s != g_system) bridge_fail("only one system is supported", 0);
    return;
  }
  if (NumberOfSystems != 1) bridge_fail("only one system is supported", 0);
  if (NumberOfComponents != 1 || Components[0].ExtraFrameworkMolecule)
    bridge_fail("only one adsorbate component is supported", 0);
  if (Framework[s].FrameworkModel == NONE || Framework[s].NumberOfFrameworks != 1)
    bridge_fail("only one rigid framework is supported", 0);
  if (UseReplicas[s] || UseCellLists[s]) bridge_fail("replica cells and cell lists are not supported", 0);
  const REAL_MATRIX3x3 B = Box[s];
  if (BoundaryCondition[s] != TRICLINIC && BoundaryCondition[s] != RECTANGULAR && BoundaryCondition[s] != CUBIC)
    bridge_fail("only rectangular, cubic and triclinic boundary conditions are supported", 0);
  /* the reference also takes a cubic cell as TRICLINIC (src/framework.c:
   * 1987-1991), with off-diagonal elements of rounding size (cos 90 deg):
   * such a box goes to the orthorhombic path */
  const int tri = BoundaryCondition[s] == TRICLINIC &&
                  fabs(B.bx) + fabs(B.cx) + fabs(B.cy) > 1e-12 * (B.ax + B.by + B.cz);
  if (tri && (B.ay != 0.0 || B.az != 0.0 || B.bz != 0.0))
    bridge_fail("the triclinic box must have a along x and b in the xy plane", 0);
  if (ChargeMethod != NONE && ChargeMethod != EWALD) bridge_fail("charges need the Ewald method", 0);
  if (ChargeMethod == EWALD && (OmitEwaldFourier || fabs(CutOffChargeChargeSquared[s] - CutOffVDWSquared) > 1e-12))
    bridge_fail("Ewald needs its Fourier part and one cut-off for VDW and charges", 0);

  const int nt = NumberOfPseudoAtoms, c = 0;
  if (nt > BRIDGE_MAXTYPES) bridge_fail("too many pseudo-atom types", 0);
  const COMPONENT *C = &Components[c];
  double *eps = calloc((size_t)nt * nt, sizeof(double)), *sig2 = calloc((size_t)nt * nt, sizeof(double));
  double *shift = calloc((size_t)nt * nt, sizeof(double));
  for (int a = 0; a < nt; a++)
    for (int b = 0; b < nt; b++) {
      const int t = PotentialType[a][b];
      if (t == LENNARD_JONES) {
        eps[a * nt + b] = PotentialParms[a][b][0];
        sig2[a * nt + b] = PotentialParms[a][b][1] * PotentialParms[a][b][1];
        shift[a * nt + b] = PotentialParms[a][b][2];   /* ComputePotentialShifts, src/potentials.c:5263 */
      } else if (t != ZERO_POTENTIAL && t != UNDEFINED_POTENTIAL) {
        bridge_fail("only Lennard-Jones potentials are supported", 0);
      }
    }
  const int nfw = Framework[s].NumberOfAtoms[0];
  double *fx = malloc(sizeof(double) * 3 * (size_t)nfw), *fq = malloc(sizeof(double) * (size_t)nfw);
  int *ft = malloc(sizeof(int) * (size_t)nfw);
  for (int i = 0; i < nfw; i++) {
    const ATOM *A = &Framework[s].Atoms[0][i];
    fx[3 * i] = A->Position.x;
    fx[3 * i + 1] = A->Position.y;
    fx[3 * i + 2] = A->Position.z;
    ft[i] = A->Type;
    fq[i] = A->Charge;
  }
  g_natom = C->NumberOfAtoms;
  if (g_natom > 64) bridge_fail("molecules of more than 64 atoms are not supported", 0);
  double *ref = malloc(sizeof(double) * 3 * (size_t)g_natom);
  for (int a = 0; a < g_natom; a++) {
    ref[3 * a] = C->Positions[a].x;
    ref[3 * a + 1] = C->Positions[a].y;
    ref[3 * a + 2] = C->Positions[a].z;
  }
  for (int t = 0; t < BRIDGE_MAXTYPES; t++) g_atom_of_type[t] = -1;
  for (int a = g_natom - 1; a >= 0; a--) g_atom_of_type[C->Type[a]] = a;

  rgpu_system_desc d;
  memset(&d, 0, sizeof d);
  d.box[0] = B.ax;
  d.box[1] = B.by;
  d.box[2] = B.cz;
  if (tri) {
    /* the box matrix, row-major, columns a, b, c (Box[], src/framework.c:2025-2040) */
    const double m[9] = {B.ax, B.bx, B.cx, B.ay, B.by, B.cy, B.az, B.bz, B.cz};
    for (int i = 0; i < 9; i++) d.cell_matrix[i] = m[i];
    d.box[0] = sqrt(B.ax * B.ax);
    d.box[1] = sqrt(B.bx * B.bx + B.by * B.by);
    d.box[2] = sqrt(B.cx * B.cx + B.cy * B.cy + B.cz * B.cz);
  }
  d.cutoff = sqrt(CutOffVDWSquared);
  d.beta = Beta[s];
  d.coulomb = COULOMBIC_CONVERSION_FACTOR;
  d.overlap = EnergyOverlapCriteria;
  d.nfw = nfw;
  d.fw_xyz = fx;
  d.fw_type = ft;
  d.fw_q = fq;
  d.ntypes = nt;
  d.eps = eps;
  d.sig2 = sig2;
  d.shift = shift;
  d.natom = g_natom;
  d.mol_type = C->Type;
  d.mol_q = C->Charge;
  d.mol_ref = ref;
  d.start_bead = C->StartingBead;
  d.ewald = ChargeMethod == EWALD;
  d.alpha = d.ewald ? Alpha[s] : 0.0;
  if (d.ewald) {
    d.kmax[0] = kvec[s].x;
    d.kmax[1] = kvec[s].y;
    d.kmax[2] = kvec[s].z;
  }
  d.maxmol = BRIDGE_MAXMOL;
  for (int k = 0; k < 6; k++) d.move_cum[k] = 1.0;   /* the engine is not used */
  d.max_translation = 1.0;
  d.max_rotation = 1.0;
  d.fugacity_beta_v = 1.0;
  d.ntrial_first = d.ntrial = 1;
  const int rc = rgpu_system_create(&g_sys, &d);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_system_create", rc);
  if (Framework[s].FrameworkModel == GRID) bridge_grids(C, s);
  free(eps);
  free(sig2);
  free(shift);
  free(fx);
  free(fq);
  free(ft);
  free(ref);
  g_system = s;
  g_comp = c;
  g_mirror = malloc(sizeof(double) * 3 * (size_t)g_natom * BRIDGE_MAXMOL);
  g_scratch = malloc(sizeof(double) * 3 * (size_t)g_natom * BRIDGE_MAXMOL);
  const char *p = getenv("RASPA_GPU_PRECISION");
  g_prec = (p && !strcmp(p, "mixed")) ? RGPU_MIXED : RGPU_FP64;
  if (getenv("RASPA_GPU_BRIDGE_STATS")) atexit(print_stats);
}

/* cached results of the last point and of the last move */
static struct {
  int valid, type, exclude;
  double p[3], e[4];
} g_pt;
static struct {
  int valid, m, ov;
  double x[3 * 64], d[4];
} g_mv;

/* uploads Adsorbates[][] when it differs from the device's copy */
static void bridge_sync(void)
{
  bridge_init();
  const int s = g_system, n = NumberOfAdsorbateMolecules[s];
  if (n > BRIDGE_MAXMOL) bridge_fail("more adsorbate molecules than the bridge holds", 0);
  double *x = g_scratch;
  for (int j = 0; j < n; j++) {
    if (Adsorbates[s][j].Type != g_comp) bridge_fail("unexpected adsorbate component", 0);
    for (int a = 0; a < g_natom; a++) {
      const POINT P = Adsorbates[s][j].Atoms[a].Position;
      double *o = x + 3 * ((size_t)j * g_natom + a);
      o[0] = P.x;
      o[1] = P.y;
      o[2] = P.z;
    }
  }
  const size_t bytes = sizeof(double) * 3 * (size_t)g_natom * n;
  if (n == g_mirror_n && !memcmp(x, g_mirror, bytes)) return;
  const int rc = rgpu_set_adsorbates(g_sys, n, x);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_set_adsorbates", rc);
  memcpy(g_mirror, x, bytes);
  g_mirror_n = n;
  g_pt.valid = g_mv.valid = 0;
  g_pending_store = -1;
  g_calls[3]++;
}

/* {host VDW, host charge, adsorbate VDW, adsorbate charge} of a bead of
 * pseudo-atom `type` at p, leaving out adsorbate molecule `exclude` */
static const double *point_energies(POINT p, int type, int exclude)
{
  bridge_sync();
  if (exclude < 0 || exclude >= g_mirror_n) exclude = -1;
  if (g_pt.valid && g_pt.type == type && g_pt.exclude == exclude && g_pt.p[0] == p.x && g_pt.p[1] == p.y &&
      g_pt.p[2] == p.z)
    return g_pt.e;
  if (type < 0 || type >= BRIDGE_MAXTYPES || g_atom_of_type[type] < 0)
    bridge_fail("pseudo-atom not in the adsorbate", 0);
  const double xyz[3] = {p.x, p.y, p.z};
  const int atom = g_atom_of_type[type];
  const int rc = rgpu_bead_energies(g_sys, g_prec, 1, xyz, &atom, &exclude, g_pt.e);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_bead_energies", rc);
  g_pt.valid = 1;
  g_pt.type = type;
  g_pt.exclude = exclude;
  g_pt.p[0] = p.x;
  g_pt.p[1] = p.y;
  g_pt.p[2] = p.z;
  g_calls[0]++;
  return g_pt.e;
}

REAL __wrap_CalculateFrameworkVDWEnergyAtPosition(POINT posA, int typeA, REAL scaling)
{
  if (scaling != 1.0) bridge_fail("CFCMC scaling is not supported", 0);
  return point_energies(posA, typeA, CurrentAdsorbateMolecule)[0];
}

void __wrap_CalculateFrameworkChargeEnergyAtPosition(POINT posA, int typeA, REAL *UChargeCharge,
                                                      REAL *UChargeBondDipole, REAL scaling)
{
  *UChargeCharge = 0.0;
  *UChargeBondDipole = 0.0;
  if (ChargeMethod == NONE || !PseudoAtoms[typeA].HasCharges) return;
  if (scaling != 1.0) bridge_fail("CFCMC scaling is not supported", 0);
  *UChargeCharge = point_energies(posA, typeA, CurrentAdsorbateMolecule)[1];
}

REAL __wrap_CalculateInterVDWEnergyAdsorbateAtPosition(POINT posA, int typeA, int exclude, REAL scaling)
{
  if (scaling != 1.0) bridge_fail("CFCMC scaling is not supported", 0);
  return point_energies(posA, typeA, exclude)[2];
}

/* the reference passes the bead's (scaled) charge as the last argument
 * (src/cbmc.c:692) */
int __wrap_CalculateInterChargeEnergyAdsorbateAtPosition(POINT posA, int typeA, REAL *UChargeCharge,
                                                         REAL *UChargeBondDipole, int exclude, REAL chargeA)
{
  *UChargeCharge = 0.0;
  *UChargeBondDipole = 0.0;
  if (ChargeMethod == NONE) return 0;
  bridge_init();
  const int a = (typeA >= 0 && typeA < BRIDGE_MAXTYPES) ? g_atom_of_type[typeA] : -1;
  if (a < 0 || chargeA != Components[g_comp].Charge[a]) bridge_fail("charge scaling is not supported", 0);
  *UChargeCharge = point_energies(posA, typeA, exclude)[3];
  return 0;
}

/* the four differences of molecule m moved to TrialPosition (both New and
 * Old, as translation and rotation call them) */
static const double *move_differences(int m, int comp, int New, int Old)
{
  bridge_sync();
  if (!New || !Old || comp != g_comp) bridge_fail("only New-and-Old differences of the adsorbate are supported", 0);
  if (m < 0 || m >= g_mirror_n) bridge_fail("molecule index out of range", 0);
  double x[3 * 64];
  for (int a = 0; a < g_natom; a++) {
    const POINT P = TrialPosition[g_system][a];
    x[3 * a] = P.x;
    x[3 * a + 1] = P.y;
    x[3 * a + 2] = P.z;
  }
  if (g_mv.valid && g_mv.m == m && !memcmp(g_mv.x, x, sizeof(double) * 3 * g_natom)) return g_mv.d;
  const int rc = rgpu_move_energy_difference(g_sys, g_prec, m, x, g_mv.d, &g_mv.ov);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_move_energy_difference", rc);
  memcpy(g_mv.x, x, sizeof(double) * 3 * g_natom);
  g_mv.m = m;
  g_mv.valid = 1;
  g_calls[1]++;
  return g_mv.d;
}

/* an overlap anywhere in the move rejects it; the reference stops at the
 * first routine whose pairs overlap, with the same outcome */
int __wrap_CalculateInterVDWEnergyDifferenceAdsorbate(int m, int comp, int New, int Old)
{
  const double *d = move_differences(m, comp, New, Old);
  UAdsorbateVDWDelta[g_system] = d[2];
  return OVERLAP = g_mv.ov ? TRUE : FALSE;
}

int __wrap_CalculateInterChargeChargeEnergyDifferenceAdsorbate(int m, int comp, int New, int Old)
{
  const double *d = move_differences(m, comp, New, Old);
  UAdsorbateChargeChargeRealDelta[g_system] = ChargeMethod == NONE ? 0.0 : d[3];
  return OVERLAP = g_mv.ov ? TRUE : FALSE;
}

int __wrap_CalculateFrameworkAdsorbateVDWEnergyDifference(int m, int comp, int New, int Old, int CanUseGridNew,
                                                          int CanUseGridOld)
{
  (void)CanUseGridNew;
  (void)CanUseGridOld;
  const double *d = move_differences(m, comp, New, Old);
  UHostVDWDelta[g_system] = d[0];
  return OVERLAP = g_mv.ov ? TRUE : FALSE;
}

int __wrap_CalculateFrameworkAdsorbateChargeChargeEnergyDifference(int m, int comp, int New, int Old,
                                                                   int CanUseGridNew, int CanUseGridOld)
{
  (void)CanUseGridNew;
  (void)CanUseGridOld;
  const double *d = move_differences(m, comp, New, Old);
  UHostChargeChargeRealDelta[g_system] = ChargeMethod == NONE ? 0.0 : d[1];
  return OVERLAP = g_mv.ov ? TRUE : FALSE;
}

int __wrap_CalculateEwaldFourierAdsorbate(int NewMolecule, int OldMolecule, int mol, int store)
{
  const int s = CurrentSystem;
  NetChargeAdsorbateDelta = 0.0;
  UAdsorbateAdsorbateChargeChargeFourierDelta[s] = UAdsorbateCationChargeChargeFourierDelta[s] = 0.0;
  UHostAdsorbateChargeChargeFourierDelta[s] = UHostCationChargeChargeFourierDelta[s] = 0.0;
  UCationCationChargeChargeFourierDelta[s] = 0.0;
  UAdsorbateAdsorbateChargeBondDipoleFourierDelta[s] = UAdsorbateCationChargeBondDipoleFourierDelta[s] = 0.0;
  UHostAdsorbateChargeBondDipoleFourierDelta[s] = UHostCationChargeBondDipoleFourierDelta[s] = 0.0;
  UCationCationChargeBondDipoleFourierDelta[s] = 0.0;
  UAdsorbateAdsorbateBondDipoleBondDipoleFourierDelta[s] = UAdsorbateCationBondDipoleBondDipoleFourierDelta[s] = 0.0;
  UHostAdsorbateBondDipoleBondDipoleFourierDelta[s] = UHostCationBondDipoleBondDipoleFourierDelta[s] = 0.0;
  UCationCationBondDipoleBondDipoleFourierDelta[s] = 0.0;
  if (ChargeMethod != EWALD || OmitEwaldFourier) return 0;
  bridge_sync();
  double x[3 * 64], out[3];
  if (NewMolecule)
    for (int a = 0; a < g_natom; a++) {
      x[3 * a] = TrialPosition[s][a].x;
      x[3 * a + 1] = TrialPosition[s][a].y;
      x[3 * a + 2] = TrialPosition[s][a].z;
    }
  if (OldMolecule && (mol < 0 || mol >= g_mirror_n)) bridge_fail("molecule index out of range", 0);
  const int rc = rgpu_ewald_fourier_difference(g_sys, g_prec, OldMolecule ? mol : -1, NewMolecule ? x : NULL, out);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_ewald_fourier_difference", rc);
  UAdsorbateAdsorbateChargeChargeFourierDelta[s] = out[0];
  UHostAdsorbateChargeChargeFourierDelta[s] = out[1];
  NetChargeAdsorbateDelta = out[2];
  g_pending_store = store;
  g_calls[2]++;
  return 0;
}

void __wrap_AcceptEwaldAdsorbateMove(int A)
{
  if (ChargeMethod != EWALD || OmitEwaldFourier) return;
  if (A != g_pending_store) bridge_fail("accepted an Ewald candidate that is not on the device", 0);
  const int rc = rgpu_ewald_accept(g_sys);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_ewald_accept", rc);
  g_pending_store = -1;
}

/* MakeGrid (src/grids.c:431-690), the MAKE_GRID simulation type: the VDW
 * grid of every pseudo-atom of GridTypeList and, with Ewald charges, the
 * Coulomb grid of a unit charge are built on the GPU (rgpu_grid_build,
 * rgpu_grid_build_coulomb) over the unit cell, with the reference's point
 * counts (odd, from the spacings), and written where and as WriteVDWGrid and
 * WriteCoulombGrid write them (rgpu_grid_write_file). The grids agree with
 * the reference's to FP32 rounding (the framework sums run in another
 * order). */
static float *bridge_grid_buffer(const int n[3])
{
  float *d = NULL;
  const size_t bytes = sizeof(float) * 8 * (size_t)(n[0] + 1) * (n[1] + 1) * (n[2] + 1);
  if (cudaMalloc((void **)&d, bytes) != cudaSuccess) bridge_fail("cudaMalloc of a grid", 0);
  return d;
}

void __wrap_MakeGrid(void)
{
  bridge_init();
  const int s = CurrentSystem;
  const REAL_MATRIX3x3 U = UnitCellBox[s];
  /* the enclosing box of the unit cell (src/grids.c:336-360) */
  double size[3] = {0.0, 0.0, 0.0}, shift[3] = {0.0, 0.0, 0.0};
  const double vec[3][3] = {{U.ax, U.ay, U.az}, {U.bx, U.by, U.bz}, {U.cx, U.cy, U.cz}};
  for (int v = 0; v < 3; v++)
    for (int c = 0; c < 3; c++) {
      size[c] += fabs(vec[v][c]);
      if (vec[v][c] < 0.0) shift[c] += vec[v][c];
    }
  rgpu_grid_file_header h;
  memset(&h, 0, sizeof h);
  for (int c = 0; c < 3; c++) {
    h.size[c] = size[c];
    h.shift[c] = shift[c];
  }
  h.unit_cell[0] = UnitCellSize[s].x;
  h.unit_cell[1] = UnitCellSize[s].y;
  h.unit_cell[2] = UnitCellSize[s].z;
  h.unit_cells[0] = NumberOfUnitCells[s].x;
  h.unit_cells[1] = NumberOfUnitCells[s].y;
  h.unit_cells[2] = NumberOfUnitCells[s].z;
  /* point counts: size / spacing, made odd (:486-492, :588-594) */
  int n[3];
  for (int c = 0; c < 3; c++) {
    n[c] = (int)(size[c] / SpacingVDWGrid);
    if (n[c] % 2 == 0) n[c]++;
    h.npts[c] = n[c];
    h.delta[c] = size[c] / (double)n[c];
  }
  NumberOfVDWGridPoints.x = n[0];
  NumberOfVDWGridPoints.y = n[1];
  NumberOfVDWGridPoints.z = n[2];
  h.spacing = SpacingVDWGrid;
  char path[4096];
  float *d = bridge_grid_buffer(n);
  for (int l = 0; l < NumberOfGrids; l++) {
    const int type = GridTypeList[l];
    fprintf(OutputFilePtr[s], "Creating grid %d [%s] on the GPU\n", l, PseudoAtoms[type].Name);
    fflush(OutputFilePtr[s]);
    int rc = rgpu_grid_build(g_sys, type, n, size, shift, d);
    if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_build", rc);
    rc = rgpu_grid_file_path(path, sizeof path, RASPA_DIRECTORY, ForceField, Framework[s].Name[0], SpacingVDWGrid,
                             PseudoAtoms[type].Name, ShiftPotentials, NULL);
    if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_file_path", rc);
    rc = rgpu_grid_write_file(path, 0, &h, d);
    if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_write_file", rc);
  }
  cudaFree(d);
  if (ChargeMethod != EWALD) {
    /* the reference's MakeGrid ends the program here without charges (:611-614) */
    fprintf(stderr, "Skipping the Coulombic grid\n");
    exit(0);
  }
  for (int c = 0; c < 3; c++) {
    n[c] = (int)(size[c] / SpacingCoulombGrid);
    if (n[c] % 2 == 0) n[c]++;
    h.npts[c] = n[c];
    h.delta[c] = size[c] / (double)n[c];
  }
  h.spacing = SpacingCoulombGrid;
  h.ewald_precision = EwaldPrecision;
  fprintf(OutputFilePtr[s], "Creating the Ewald-Coulomb grid on the GPU (%d x %d x %d)\n", n[0], n[1], n[2]);
  fflush(OutputFilePtr[s]);
  d = bridge_grid_buffer(n);
  int rc = rgpu_grid_build_coulomb(g_sys, n, size, shift, d);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_build_coulomb", rc);
  const int nc[3] = {NumberOfUnitCells[s].x, NumberOfUnitCells[s].y, NumberOfUnitCells[s].z};
  rc = rgpu_grid_file_path(path, sizeof path, RASPA_DIRECTORY, ForceField, Framework[s].Name[0], SpacingCoulombGrid,
                           NULL, ShiftPotentials, nc);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_file_path", rc);
  rc = rgpu_grid_write_file(path, 1, &h, d);
  if (rc != RGPU_SUCCESS) bridge_fail("rgpu_grid_write_file", rc);
  cudaFree(d);
}
