/* Golden-vector harness around the reference's own energy routines.
 *
 * TEST INFRASTRUCTURE ONLY. It is linked against the reference's src/*.c
 * (built by oracle/Makefile into oracle/_ref/) and is run in this container
 * by tests/golden/make_golden.py to produce the committed fixtures. Nothing in
 * the product links or runs it.
 *
 * Usage:  ref_harness <run-directory> <commands-file> <output-file>
 *
 * The run directory holds a RASPA input written by raspa2_b200.raspa_io
 * (simulation.input, <name>.cif, pseudo_atoms.def,
 * force_field_mixing_rules.def, <molecule>.def). The harness reads it with the
 * reference's ReadInputFile (src/input.c), then executes one command per line:
 *
 *   system                 dump box, constants, pseudo-atoms, framework atoms
 *   insert x0 y0 z0 ...    InsertAdsorbateMolecule (src/molecule.c:3075) at
 *                          the given atom positions (component 0)
 *   energy                 CalculateEnergy (src/integration.c:250) totals
 *   point T x y z excl     Calculate{Framework,Inter}{VDW,Charge}EnergyAtPosition
 *                          (src/framework_energy.c:60,176; src/inter_energy.c:321,393)
 *   move m x0 y0 z0 ...    the translation/rotation energy differences of
 *                          src/mc_moves.c:1601-1629 for molecule m moved to
 *                          the given positions (no acceptance)
 *   accept m x0 ...        as `move`, then accept it (src/mc_moves.c:1740-1748)
 *   ewald_insert x0 ...    CalculateEwaldFourierAdsorbate(TRUE,FALSE,N,0) -> "fourier"
 *   ewald_delete m         CalculateEwaldFourierAdsorbate(FALSE,TRUE,m,0)
 *   cbmc_insert seed       GrowMolecule(CBMC_INSERTION) (src/cbmc.c:3056) after
 *                          seeding the reference RNG (src/utils.c:324)
 *   cbmc_delete m seed     RetraceMolecule(CBMC_DELETION) (src/cbmc.c:2928)
 *   deriv T x y z          CalculateDerivativesAtPositionVDW
 *                          (src/framework_hessian.c:63)
 *   interp T x y z         InterpolateVDWGrid (src/grids.c:979); needs
 *                          UseTabularGrid and a grid file in the run directory
 *   derivreal x y z        CalculateDerivativesAtPositionReal
 *                          (src/framework_hessian.c:111), unit probe charge;
 *                          prints the smallest distance last
 *   interpc T x y z        InterpolateCoulombGrid (src/grids.c:1200) for
 *                          pseudo-atom T (its charge times the grid value)
 *   makegrid               MakeGrid (src/grids.c:431); writes the grid files
 *                          and (as the reference does) ends the process
 *
 * Every result line is "<tag> <values...>" with values printed %.17g.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdbool.h>
#include <unistd.h>
#include <math.h>

#include "constants.h"
#include "simulation.h"
#include "molecule.h"
#include "framework.h"
#include "framework_energy.h"
#include "inter_energy.h"
#include "ewald.h"
#include "potentials.h"
#include "cbmc.h"
#include "mc_moves.h"
#include "grids.h"
#include "input.h"
#include "integration.h"
#include "utils.h"
#include "framework_hessian.h"
#include "run.h"
#include "thermo_baro_stats.h"
#include "equations_of_state.h"
#include "statistics.h"
#include "output.h"

extern bool STREAM;
extern char *INPUT_CRYSTAL;

static FILE *out;

static void p1(const char *tag, int n, const double *v)
{
  fprintf(out, "%s", tag);
  for (int i = 0; i < n; i++) fprintf(out, " %.17g", v[i]);
  fprintf(out, "\n");
}

static int parse_doubles(char *s, double *v, int max)
{
  int n = 0;
  char *tok = strtok(s, " \t\n");
  while (tok && n < max) { v[n++] = atof(tok); tok = strtok(NULL, " \t\n"); }
  return n;
}

static void set_trial(const double *v, int n_atoms)
{
  for (int i = 0; i < n_atoms; i++) {
    TrialPosition[CurrentSystem][i].x = v[3 * i + 0];
    TrialPosition[CurrentSystem][i].y = v[3 * i + 1];
    TrialPosition[CurrentSystem][i].z = v[3 * i + 2];
    TrialAnisotropicPosition[CurrentSystem][i] = TrialPosition[CurrentSystem][i];
    /* InsertAdsorbateMolecule copies NewPosition (src/molecule.c:3136) */
    NewPosition[CurrentSystem][i] = TrialPosition[CurrentSystem][i];
    CFVDWScaling[i] = 1.0;
    CFChargeScaling[i] = 1.0;
  }
}

static void dump_system(void)
{
  double v[16];
  v[0] = Box[0].ax; v[1] = Box[0].ay; v[2] = Box[0].az;
  v[3] = Box[0].bx; v[4] = Box[0].by; v[5] = Box[0].bz;
  v[6] = Box[0].cx; v[7] = Box[0].cy; v[8] = Box[0].cz;
  p1("box", 9, v);
  v[0] = Volume[0]; p1("volume", 1, v);
  v[0] = COULOMBIC_CONVERSION_FACTOR; v[1] = KELVIN_TO_ENERGY; v[2] = ENERGY_TO_KELVIN;
  v[3] = K_B; v[4] = Beta[0]; v[5] = EnergyOverlapCriteria; v[6] = MinimumRosenbluthFactor;
  v[7] = CutOffVDWSquared; v[8] = CutOffChargeChargeSquared[0];
  p1("constants", 9, v);
  v[0] = ChargeMethod == EWALD ? Alpha[0] : 0.0;
  v[1] = kvec[0].x; v[2] = kvec[0].y; v[3] = kvec[0].z;
  v[4] = ChargeMethod == EWALD ? NumberOfKVectors[0] : 0;
  v[5] = ChargeMethod == EWALD ? ReciprocalCutOffSquared[0] : 0.0;
  v[6] = UIon[0]; v[7] = NetChargeFramework[0];
  p1("ewald", 8, v);
  v[0] = UseReplicas[0]; v[1] = NumberOfReplicaCells[0].x; v[2] = NumberOfReplicaCells[0].y;
  v[3] = NumberOfReplicaCells[0].z; v[4] = NumberOfUnitCells[0].x; v[5] = NumberOfUnitCells[0].y;
  v[6] = NumberOfUnitCells[0].z; v[7] = UseCellLists[0]; v[8] = BoundaryCondition[0];
  p1("replicas", 9, v);
  fprintf(out, "npseudo %d\n", NumberOfPseudoAtoms);
  for (int i = 0; i < NumberOfPseudoAtoms; i++) {
    fprintf(out, "pseudo %d %s %.17g %d\n", i, PseudoAtoms[i].Name, PseudoAtoms[i].Charge1,
            (int)PseudoAtoms[i].HasCharges);
  }
  for (int i = 0; i < NumberOfPseudoAtoms; i++)
    for (int j = 0; j < NumberOfPseudoAtoms; j++)
      if (PotentialType[i][j] == LENNARD_JONES)
        fprintf(out, "lj %d %d %.17g %.17g %.17g\n", i, j, PotentialParms[i][j][0],
                PotentialParms[i][j][1], PotentialParms[i][j][2]);
  int nf = Framework[0].TotalNumberOfAtoms;
  fprintf(out, "nframework %d\n", nf);
  for (int f = 0; f < Framework[0].NumberOfFrameworks; f++)
    for (int i = 0; i < Framework[0].NumberOfAtoms[f]; i++) {
      ATOM *a = &Framework[0].Atoms[f][i];
      fprintf(out, "fw %.17g %.17g %.17g %d %.17g\n", a->Position.x, a->Position.y,
              a->Position.z, a->Type, a->Charge);
    }
  COMPONENT *c = &Components[0];
  fprintf(out, "component %d %d\n", c->NumberOfAtoms, c->StartingBead);
  for (int i = 0; i < c->NumberOfAtoms; i++)
    fprintf(out, "catom %d %.17g %.17g %.17g %.17g\n", c->Type[i], c->Positions[i].x,
            c->Positions[i].y, c->Positions[i].z, c->Charge[i]);
  v[0] = NumberOfTrialPositionsSwap; v[1] = NumberOfTrialPositionsForTheFirstBeadSwap;
  v[2] = BiasingMethod; v[3] = c->IdealGasRosenbluthWeight[0];
  v[4] = c->FugacityCoefficient[0]; v[5] = c->PartialPressure[0];
  p1("mcparams", 6, v);
}

static void print_energy(void)
{
  double v[12];
  CalculateEnergy();
  v[0] = UHostAdsorbateVDW[0];
  v[1] = UAdsorbateAdsorbateVDW[0];
  v[2] = UHostAdsorbateChargeChargeReal[0];
  v[3] = UAdsorbateAdsorbateChargeChargeReal[0];
  v[4] = UHostAdsorbateChargeChargeFourier[0];
  v[5] = UAdsorbateAdsorbateChargeChargeFourier[0];
  v[6] = UTotal[0];
  v[7] = NumberOfAdsorbateMolecules[0];
  v[8] = UTailCorrection[0];
  p1("energy", 9, v);
}

static void clear_deltas(void)
{
  UHostVDWDelta[0] = UAdsorbateVDWDelta[0] = 0.0;
  UHostChargeChargeRealDelta[0] = UAdsorbateChargeChargeRealDelta[0] = 0.0;
  UHostAdsorbateChargeChargeFourierDelta[0] = UAdsorbateAdsorbateChargeChargeFourierDelta[0] = 0.0;
}

static int do_move(int m)
{
  /* the order and early-outs of src/mc_moves.c:1601-1629 */
  clear_deltas();
  OVERLAP = FALSE;
  CurrentAdsorbateMolecule = m;
  CurrentCationMolecule = -1;
  CalculateInterVDWEnergyDifferenceAdsorbate(m, 0, TRUE, TRUE);
  if (OVERLAP) return 1;
  CalculateInterChargeChargeEnergyDifferenceAdsorbate(m, 0, TRUE, TRUE);
  if (OVERLAP) return 1;
  CalculateFrameworkAdsorbateVDWEnergyDifference(m, 0, TRUE, TRUE, TRUE, TRUE);
  if (OVERLAP) return 1;
  CalculateFrameworkAdsorbateChargeChargeEnergyDifference(m, 0, TRUE, TRUE, TRUE, TRUE);
  if (OVERLAP) return 1;
  if (ChargeMethod == EWALD) CalculateEwaldFourierAdsorbate(TRUE, TRUE, m, 0);
  return 0;
}

static void print_deltas(const char *tag, int ov)
{
  double v[8];
  v[0] = ov;
  v[1] = UHostVDWDelta[0];
  v[2] = UAdsorbateVDWDelta[0];
  v[3] = UHostChargeChargeRealDelta[0];
  v[4] = UAdsorbateChargeChargeRealDelta[0];
  v[5] = UHostAdsorbateChargeChargeFourierDelta[0];
  v[6] = UAdsorbateAdsorbateChargeChargeFourierDelta[0];
  v[7] = NetChargeAdsorbateDelta;
  p1(tag, 8, v);
}

static void print_cbmc(const char *tag, double w, int n_atoms, int new_)
{
  double v[8 + 3 * 16];
  int k = 0;
  v[k++] = OVERLAP;
  v[k++] = w;
  v[k++] = new_ ? UHostVDWNew[0] : UHostVDWOld[0];
  v[k++] = new_ ? UAdsorbateVDWNew[0] : UAdsorbateVDWOld[0];
  v[k++] = new_ ? UHostChargeChargeNew[0] : UHostChargeChargeOld[0];
  v[k++] = new_ ? UAdsorbateChargeChargeNew[0] : UAdsorbateChargeChargeOld[0];
  for (int i = 0; i < n_atoms && new_; i++) {
    v[k++] = NewPosition[0][i].x; v[k++] = NewPosition[0][i].y; v[k++] = NewPosition[0][i].z;
  }
  /* the next draw of the reference stream: checks how many numbers were consumed */
  v[k++] = RandomNumber();
  p1(tag, k, v);
}

int main(int argc, char **argv)
{
  if (argc < 4) { fprintf(stderr, "usage: ref_harness dir commands out\n"); return 2; }
  char cmdpath[4096], outpath[4096];
  /* resolve the command and output paths before changing directory */
  if (!realpath(argv[2], cmdpath)) { perror("commands"); return 2; }
  snprintf(outpath, sizeof outpath, "%s", argv[3]);
  if (outpath[0] != '/') {
    char cwd[2048];
    if (!getcwd(cwd, sizeof cwd)) return 2;
    snprintf(outpath, sizeof outpath, "%s/%s", cwd, argv[3]);
  }
  if (chdir(argv[1]) != 0) { perror("chdir"); return 2; }
  char rundir[2048];
  if (!getcwd(rundir, sizeof rundir)) return 2;

  RASPA_DIRECTORY = strdup(rundir);
  INPUT_CRYSTAL = strdup("");
  STREAM = false;
  ReadInputFile("simulation.input");

  out = fopen(outpath, "w");
  if (!out) { perror("out"); return 2; }
  FILE *cmds = fopen(cmdpath, "r");
  if (!cmds) { perror("cmds"); return 2; }

  CurrentSystem = 0;
  CurrentComponent = 0;
  CurrentIsothermPressure = 0;
  ComputeGasPropertiesForAllSystems();
  InitializesEnergiesAllSystems();
  CalculateTotalEnergyAllSystems();
  CurrentSystem = 0;
  CurrentComponent = 0;

  static char line[1 << 16];
  static double v[4096];
  int n_atoms = Components[0].NumberOfAtoms;
  while (fgets(line, sizeof line, cmds)) {
    char cmd[64];
    if (sscanf(line, "%63s", cmd) != 1) continue;
    char *rest = line + strlen(cmd);
    if (!strcmp(cmd, "system")) {
      dump_system();
    } else if (!strcmp(cmd, "insert")) {
      int n = parse_doubles(rest, v, 4096);
      if (n != 3 * n_atoms) { fprintf(stderr, "insert: need %d values\n", 3 * n_atoms); return 3; }
      set_trial(v, n_atoms);
      CurrentComponent = 0;
      CurrentAdsorbateMolecule = NumberOfAdsorbateMolecules[0];
      InsertAdsorbateMolecule();
    } else if (!strcmp(cmd, "energy")) {
      print_energy();
    } else if (!strcmp(cmd, "point")) {
      int n = parse_doubles(rest, v, 8);
      if (n < 5) return 3;
      int type = (int)v[0], excl = (int)v[4];
      POINT p = {v[1], v[2], v[3]};
      double r[5];
      REAL ucc = 0, ubd = 0, iucc = 0, iubd = 0;
      r[0] = CalculateFrameworkVDWEnergyAtPosition(p, type, 1.0);
      CalculateFrameworkChargeEnergyAtPosition(p, type, &ucc, &ubd, 1.0);
      r[1] = ucc;
      r[2] = CalculateInterVDWEnergyAdsorbateAtPosition(p, type, excl, 1.0);
      CalculateInterChargeEnergyAdsorbateAtPosition(p, type, &iucc, &iubd, excl,
                                                    PseudoAtoms[type].Charge1);
      r[3] = iucc;
      p1("point", 4, r);
    } else if (!strcmp(cmd, "move") || !strcmp(cmd, "accept")) {
      int n = parse_doubles(rest, v, 4096);
      int m = (int)v[0];
      if (n != 1 + 3 * n_atoms) return 3;
      set_trial(v + 1, n_atoms);
      int ov = do_move(m);
      print_deltas("move", ov);
      if (!strcmp(cmd, "accept") && !ov) {
        if (ChargeMethod == EWALD) AcceptEwaldAdsorbateMove(0);
        for (int i = 0; i < n_atoms; i++) {
          Adsorbates[0][m].Atoms[i].Position = TrialPosition[0][i];
          Adsorbates[0][m].Atoms[i].AnisotropicPosition = TrialAnisotropicPosition[0][i];
        }
      }
    } else if (!strcmp(cmd, "ewald_insert")) {
      int n = parse_doubles(rest, v, 4096);
      if (n != 3 * n_atoms) return 3;
      set_trial(v, n_atoms);
      clear_deltas();
      CurrentAdsorbateMolecule = NumberOfAdsorbateMolecules[0];
      CalculateEwaldFourierAdsorbate(TRUE, FALSE, NumberOfAdsorbateMolecules[0], 0);
      print_deltas("fourier", 0);
    } else if (!strcmp(cmd, "ewald_delete")) {
      int n = parse_doubles(rest, v, 8);
      if (n != 1) return 3;
      int m = (int)v[0];
      clear_deltas();
      CurrentAdsorbateMolecule = m;
      CalculateEwaldFourierAdsorbate(FALSE, TRUE, m, 0);
      print_deltas("fourier", 0);
    } else if (!strcmp(cmd, "cbmc_insert")) {
      int n = parse_doubles(rest, v, 8);
      if (n != 1) return 3;
      InitializeRandomNumberGenerator((unsigned long long)v[0]);
      CurrentComponent = 0;
      CurrentAdsorbateMolecule = NumberOfAdsorbateMolecules[0];
      CurrentCationMolecule = NumberOfCationMolecules[0];
      for (int i = 0; i < n_atoms; i++) { CFVDWScaling[i] = 1.0; CFChargeScaling[i] = 1.0; }
      NumberOfBeadsAlreadyPlaced = 0;
      int st = NumberOfTrialPositions, sf = NumberOfTrialPositionsForTheFirstBead;
      NumberOfTrialPositions = NumberOfTrialPositionsSwap;
      NumberOfTrialPositionsForTheFirstBead = NumberOfTrialPositionsForTheFirstBeadSwap;
      double w = GrowMolecule(CBMC_INSERTION);
      NumberOfTrialPositions = st; NumberOfTrialPositionsForTheFirstBead = sf;
      print_cbmc("cbmc", OVERLAP ? 0.0 : w, n_atoms, 1);
    } else if (!strcmp(cmd, "cbmc_delete")) {
      int n = parse_doubles(rest, v, 8);
      if (n != 2) return 3;
      int m = (int)v[0];
      InitializeRandomNumberGenerator((unsigned long long)v[1]);
      CurrentComponent = 0;
      CurrentAdsorbateMolecule = m;
      CurrentCationMolecule = -1;
      for (int i = 0; i < n_atoms; i++) { CFVDWScaling[i] = 1.0; CFChargeScaling[i] = 1.0; }
      NumberOfBeadsAlreadyPlaced = 0;
      for (int i = 0; i < n_atoms; i++) OldPosition[i] = Adsorbates[0][m].Atoms[i].Position;
      int st = NumberOfTrialPositions, sf = NumberOfTrialPositionsForTheFirstBead;
      NumberOfTrialPositions = NumberOfTrialPositionsSwap;
      NumberOfTrialPositionsForTheFirstBead = NumberOfTrialPositionsForTheFirstBeadSwap;
      double w = RetraceMolecule(CBMC_DELETION);
      NumberOfTrialPositions = st; NumberOfTrialPositionsForTheFirstBead = sf;
      print_cbmc("cbmc", OVERLAP ? 0.0 : w, n_atoms, 0);
    } else if (!strcmp(cmd, "deriv")) {
      int n = parse_doubles(rest, v, 8);
      if (n != 4) return 3;
      VECTOR p = {v[1], v[2], v[3]}, d1;
      REAL val, d3;
      REAL_MATRIX3x3 d2;
      CalculateDerivativesAtPositionVDW(p, (int)v[0], &val, &d1, &d2, &d3);
      double r[8] = {val, d1.x, d1.y, d1.z, d2.ay, d2.az, d2.bz, d3};
      p1("deriv", 8, r);
    } else if (!strcmp(cmd, "derivreal")) {
      int n = parse_doubles(rest, v, 8);
      if (n != 3) return 3;
      VECTOR p = {v[0], v[1], v[2]}, d1;
      REAL val, d3;
      REAL_MATRIX3x3 d2;
      REAL rmin = CalculateDerivativesAtPositionReal(p, 0, &val, &d1, &d2, &d3);
      double r[9] = {val, d1.x, d1.y, d1.z, d2.ay, d2.az, d2.bz, d3, rmin};
      p1("derivreal", 9, r);
    } else if (!strcmp(cmd, "interpc")) {
      int n = parse_doubles(rest, v, 8);
      if (n != 4) return 3;
      VECTOR p = {v[1], v[2], v[3]};
      double r = InterpolateCoulombGrid((int)v[0], p);
      p1("interpc", 1, &r);
    } else if (!strcmp(cmd, "interp")) {
      int n = parse_doubles(rest, v, 8);
      if (n != 4) return 3;
      VECTOR p = {v[1], v[2], v[3]};
      double r = InterpolateVDWGrid((int)v[0], p);
      p1("interp", 1, &r);
    } else if (!strcmp(cmd, "makegrid")) {
      /* the MAKE_GRID branch of run() (src/run.c:144-152) */
      fflush(out);
      OpenOutputFile();
      PrintPreSimulationStatus();
      Framework[0].FrameworkModel = FULL;
      CurrentSystem = 0;
      MakeGrid();
    } else {
      fprintf(stderr, "unknown command %s\n", cmd);
      return 3;
    }
    fflush(out);
  }
  fclose(out);
  return 0;
}
