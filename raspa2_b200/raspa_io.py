"""Writes a `System` as RASPA2 input files.

The files follow the formats the reference reads: a P1 CIF with
`_atom_site_charge` (src/framework.c CIF reader, charges taken from the file
with `UseChargesFromCIFFile yes`), a local `pseudo_atoms.def` and
`force_field_mixing_rules.def` (`Forcefield Local`), a local molecule
definition (`MoleculeDefinition Local`, layout of molecules/TraPPE/CO2.def)
and `simulation.input` with the keywords of src/input.c. They are used to run
the reference on exactly the systems the GPU engine runs.
"""
from __future__ import annotations

import os
from typing import Optional

import numpy as np

from .systems import PSEUDO_ATOMS, TYPE_ORDER, System


def write_cif(sys: System, path: str) -> None:
    a, b, c = (float(x) for x in sys.unit_cell)
    al, be, ga = (float(x) for x in sys.cell_angles)
    vol = float(np.prod(np.diag(sys.unit_cell_matrix)))
    lines = [
        f"data_{sys.name}", "",
        f"_cell_length_a    {a:.10f}",
        f"_cell_length_b    {b:.10f}",
        f"_cell_length_c    {c:.10f}",
        f"_cell_angle_alpha {al:.10g}", f"_cell_angle_beta  {be:.10g}", f"_cell_angle_gamma {ga:.10g}",
        f"_cell_volume      {vol:.10f}", "",
        f"_symmetry_cell_setting          {'triclinic' if sys.triclinic else 'orthorhombic'}",
        "_symmetry_space_group_name_Hall 'P 1'",
        "_symmetry_space_group_name_H-M  'P 1'",
        "_symmetry_Int_Tables_number     1", "",
        "loop_", "_symmetry_equiv_pos_as_xyz", " 'x,y,z'", "",
        "loop_", "_atom_site_label", "_atom_site_type_symbol",
        "_atom_site_fract_x", "_atom_site_fract_y", "_atom_site_fract_z",
        "_atom_site_charge",
    ]
    for t, f, q in zip(sys.uc_types, sys.frac, sys.uc_charges):
        lines.append(f"{t} {t} {f[0]:.12f} {f[1]:.12f} {f[2]:.12f} {q:.8f}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_pseudo_atoms(path: str) -> None:
    hdr = ("#number of pseudo atoms\n"
           f"{len(TYPE_ORDER)}\n"
           "#type      print   as    chem  oxidation   mass        charge   polarization "
           "B-factor radii  connectivity anisotropic anisotropic-type   tinker-type\n")
    rows = []
    for name in TYPE_ORDER:
        eps, sig, q, mass = PSEUDO_ATOMS[name]
        chem = "Si" if name.startswith("Si") else name[0]
        rows.append(f"{name:<10s} yes     {chem:<4s}  {chem:<4s}  0   {mass:12.6f} {q:10.6f}"
                    "   0.0   1.0   1.0   0   0   relative   0")
    with open(path, "w") as fh:
        fh.write(hdr + "\n".join(rows) + "\n")


def write_mixing_rules(path: str, shifted: bool = True) -> None:
    rows = [f"{name:<10s} lennard-jones {PSEUDO_ATOMS[name][0]:.6f} {PSEUDO_ATOMS[name][1]:.6f}"
            for name in TYPE_ORDER]
    txt = ("# general rule for shifted vs truncated\n"
           f"{'shifted' if shifted else 'truncated'}\n"
           "# general rule tailcorrections\nno\n"
           "# number of defined interactions\n"
           f"{len(rows)}\n"
           "# type interaction, parameters\n" + "\n".join(rows) + "\n"
           "# general mixing rule for Lennard-Jones\nLorentz-Berthelot\n")
    with open(path, "w") as fh:
        fh.write(txt)


def write_molecule(sys: System, path: str) -> None:
    m = sys.molecule
    tc, pc, om = m.critical
    lines = ["# critical constants: Temperature [T], Pressure [Pa], and Acentric factor [-]",
             f"{tc}", f"{pc}", f"{om}", "# Number Of Atoms", f"{m.n_atoms}",
             "# Number of groups", "1", "# group",
             "rigid" if (m.rigid or m.n_atoms == 1) else "flexible",
             "# number of atoms", f"{m.n_atoms}", "# atomic positions"]
    for i, (t, p) in enumerate(zip(m.atom_types, m.positions)):
        if m.n_atoms == 1 or not m.rigid:
            lines.append(f"{i} {t}")
        else:
            lines.append(f"{i} {t} {p[0]:.10f} {p[1]:.10f} {p[2]:.10f}")
    if not m.rigid:
        _flexible_chain_terms(m, lines)
        with open(path, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        return
    nbond = m.n_atoms - 1 if m.n_atoms > 1 else 0
    lines.append("# Chiral centers Bond  BondDipoles Bend  UrayBradley InvBend  Torsion Imp. "
                 "Torsion Bond/Bond Stretch/Bend Bend/Bend Stretch/Torsion Bend/Torsion "
                 "IntraVDW IntraCoulomb")
    lines.append(f"               0    {nbond}            0    0            0       0        0"
                 "            0         0            0         0               0            0"
                 "        0            0")
    if nbond:
        lines.append("# Bond stretch: atom n1-n2, type, parameters")
        for i in range(nbond):
            # a linear chain of rigid bonds through the reference geometry
            lines.append(f"{i} {i + 1} RIGID_BOND")
    lines += ["# Number of config moves", "0"]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def _flexible_chain_terms(m, lines) -> None:
    """Bonded terms of a linear chain: fixed bonds, harmonic bends, TraPPE
    torsions, intramolecular LJ between atoms four or more bonds apart."""
    n = m.n_atoms
    bends = [(i, i + 1, i + 2) for i in range(n - 2)]
    tors = [(i, i + 1, i + 2, i + 3) for i in range(n - 3)]
    intra = [(i, j) for i in range(n) for j in range(i + 4, n)]
    lines.append("# Chiral centers Bond  BondDipoles Bend  UrayBradley InvBend  Torsion Imp. "
                 "Torsion Bond/Bond Stretch/Bend Bend/Bend Stretch/Torsion Bend/Torsion "
                 "IntraVDW IntraCoulomb")
    lines.append(f"               0    {n - 1}            0    {len(bends)}            0       0        {len(tors)}"
                 "            0         0            0         0               0            0"
                 f"        {len(intra)}            0")
    lines.append("# Bond stretch: atom n1-n2, type, parameters")
    for i in range(n - 1):
        lines.append(f"{i} {i + 1} FIXED_BOND {m.bond}")
    lines.append("# Bond bending: atom n1-n2-n3, type, parameters")
    for a, b, c in bends:
        lines.append(f"{a} {b} {c} HARMONIC_BEND {m.bend_k} {m.bend_theta0}")
    lines.append("# Torsion n1-n2-n3-n4 type")
    for a, b, c, d in tors:
        lines.append(f"{a} {b} {c} {d} TRAPPE_DIHEDRAL " + " ".join(f"{x}" for x in m.torsion))
    lines.append("# Intra VDW: atom n1-n2")
    for i, j in intra:
        lines.append(f"{i} {j}")
    lines += ["# Number of config moves", "0"]


def simulation_input(sys: System, cycles: int = 0, init_cycles: int = 0,
                     print_every: int = 1000, seed: Optional[int] = None,
                     simulation_type: str = "MonteCarlo",
                     grid: Optional[dict] = None, extra: str = "", restart: bool = False) -> str:
    mv = sys.moves
    lines = [
        f"SimulationType                {simulation_type}",
        f"NumberOfCycles                {cycles}",
        f"NumberOfInitializationCycles  {init_cycles}",
        f"PrintEvery                    {print_every}",
        f"RestartFile                   {'yes' if restart else 'no'}",
        "Forcefield                    Local",
        f"CutOff                        {sys.cutoff}",
        f"ChargeMethod                  {'Ewald' if sys.ewald else 'None'}",
    ]
    if sys.ewald:
        kx, ky, kz = sys.kmax
        lines.append(f"EwaldParameters               {sys.alpha} {kx} {ky} {kz}")
    # The reference's swap, Widom and reinsertion moves grow with their own
    # trial counts (src/mc_moves.c:6965, :4454; defaults 10, src/input.c:352-364),
    # not with NumberOfTrialPositions: all are set to the system's counts.
    lines.append(f"NumberOfTrialPositions        {sys.trials}")
    lines.append(f"NumberOfTrialPositionsForTheFirstBead {sys.trials_first_bead}")
    for move in ("Swap", "Widom", "Reinsertion"):
        lines.append(f"NumberOfTrialPositions{move} {sys.trials}")
        lines.append(f"NumberOfTrialPositionsForTheFirstBead{move} {sys.trials_first_bead}")
    if not sys.molecule.rigid:
        lines.append(f"NumberOfTrialPositionsTorsion {sys.torsion_trials}")
    if seed is not None:
        lines.append(f"RandomSeed                    {seed}")
    if grid:
        lines.append(f"NumberOfGrids {len(grid['types'])}")
        lines.append("GridTypes " + " ".join(grid["types"]))
        lines.append(f"SpacingVDWGrid {grid['spacing']}")
        lines.append(f"SpacingCoulombGrid {grid['spacing']}")
        if grid.get("use"):
            lines.append("UseTabularGrid yes")
    lines += [
        "",
        "Framework 0",
        f"FrameworkName                 {sys.name}",
        f"UseChargesFromCIFFile         {'yes' if sys.ewald else 'no'}",
        "RemoveAtomNumberCodeFromLabel no",
        "UnitCells                     " + " ".join(str(int(x)) for x in sys.unit_cells),
        f"ExternalTemperature           {sys.temperature}",
        f"ExternalPressure              {sys.pressure}",
        "",
    ]
    comp = [
        f"Component 0 MoleculeName             {sys.molecule.name}",
        "            MoleculeDefinition       Local",
        f"            StartingBead             {sys.molecule.starting_bead}",
        f"            IdealGasRosenbluthWeight {sys.ideal_gas_rosenbluth}",
        "            FugacityCoefficient      1.0",
        f"            TranslationProbability   {mv.translation}",
    ]
    if mv.rotation > 0 and sys.molecule.n_atoms > 1:
        comp.append(f"            RotationProbability      {mv.rotation}")
    comp.append(f"            SwapProbability          {mv.swap_insert + mv.swap_delete}")
    if mv.reinsertion > 0:
        comp.append(f"            ReinsertionProbability   {mv.reinsertion}")
    if mv.widom > 0:
        comp.append(f"            WidomProbability         {mv.widom}")
    comp.append("            CreateNumberOfMolecules  0")
    return "\n".join(lines + comp) + "\n" + extra


def write_inputs(sys: System, directory: str, **kw) -> str:
    """Write all input files of `sys` into `directory`; returns the directory."""
    os.makedirs(directory, exist_ok=True)
    write_cif(sys, os.path.join(directory, f"{sys.name}.cif"))
    write_pseudo_atoms(os.path.join(directory, "pseudo_atoms.def"))
    write_mixing_rules(os.path.join(directory, "force_field_mixing_rules.def"))
    write_molecule(sys, os.path.join(directory, f"{sys.molecule.name}.def"))
    with open(os.path.join(directory, "simulation.input"), "w") as fh:
        fh.write(simulation_input(sys, **kw))
    return directory


def write_frozen_positions(path: str, mols: np.ndarray) -> None:
    """Writes molecule positions [n_mol, n_atoms, 3] for the harness."""
    mols = np.asarray(mols, float)
    with open(path, "w") as fh:
        for m in mols:
            fh.write("insert " + " ".join(f"{v:.17g}" for v in m.reshape(-1)) + "\n")
