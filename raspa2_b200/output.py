"""RASPA-compatible results: the `.data` summary of a GCMC run, and the
energy-status blocks of the reference's output.

The reference prints, per system, a post-run summary (PrintAverageTotalSystemEnergiesMC
and friends, src/statistics.c:3990-4780, through src/output.c:6482) that its
Python wrapper parses (python/output_parser.py). `summary_text` writes the
sections of that summary that a GCMC isotherm point produces, with the
reference's headings, rules, block lines and "Average ... +/- ..." lines, so
the same parser reads a result of this package:

- "Enthalpy of adsorption" [K] and [KJ/MOL] (statistics.c:4012);
- "Number of molecules", absolute and excess loading in molecules/unit cell,
  mol/kg, mg/g, cm^3(STP)/g and cm^3(STP)/cm^3 (statistics.c:4437-4490, with
  the unit factors of src/equations_of_state.c:139-147,455-467);
- "Average Widom Rosenbluth factor" and "Average Henry coefficient"
  (statistics.c:4520-4548,4749-4775).

Averages are over NR_BLOCKS = 5 blocks of the production steps, and the
error is the reference's: twice the standard deviation of the block values
(population form, statistics.c:4455-4457).

`parse_energy_status` reads one of the reference's "Current (... energy)
Energy Status" blocks (src/output.c) into a dict of energies in K.
"""
from __future__ import annotations

import dataclasses
import re
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import units
from .systems import PSEUDO_ATOMS, System

NR_BLOCKS = 5
ATM_TO_PA = 101325.0
_LINE = "\t" + "-" * 78 + "\n"


@dataclasses.dataclass
class Block:
    """Ensemble sums of one block of production steps (rgpu_system_averages)."""
    samples: float
    n: float          # sum of molecule counts
    n2: float
    u: float          # sum of total energies (internal units)
    un: float
    widom_w: float    # sum of Widom Rosenbluth weights
    widom_n: float

    @classmethod
    def from_sums(cls, sums: Sequence[float]) -> "Block":
        s = list(sums)
        return cls(s[0], s[1], s[2], s[3], s[4], s[6], s[7])

    def minus(self, other: "Block") -> "Block":
        return Block(*(a - b for a, b in zip(dataclasses.astuple(self), dataclasses.astuple(other))))


def run_blocks(engine, gpu_systems, equilibration: int, production: int, nblocks: int = NR_BLOCKS,
               stream: int = 0) -> List[List[Block]]:
    """Runs `equilibration` then `production` steps of every system in
    `engine`, reading the ensemble sums at each of `nblocks` block ends.
    Returns, per system, its `nblocks` Blocks."""
    for g in gpu_systems:
        g.set_limits(0, equilibration)
    if equilibration:
        engine.run(equilibration, stream)
    engine.sync()
    starts = [g.state()["step"] for g in gpu_systems]
    prev = [Block.from_sums(g.averages()["sums"]) for g in gpu_systems]
    out: List[List[Block]] = [[] for _ in gpu_systems]
    done = 0
    for b in range(nblocks):
        n = production * (b + 1) // nblocks - done
        engine.run(n, stream)
        engine.sync()
        done += n
        for i, g in enumerate(gpu_systems):
            cur = Block.from_sums(g.averages()["sums"])
            out[i].append(cur.minus(prev[i]))
            prev[i] = cur
    for g, s0 in zip(gpu_systems, starts):
        assert g.state()["step"] == s0 + production
    return out


def framework_mass(sysm: System) -> float:
    """Mass of the framework in the simulation box [g/mol]."""
    per_cell = sum(PSEUDO_ATOMS[t][3] for t in sysm.uc_types)
    return per_cell * float(np.prod(sysm.unit_cells))


def molecule_mass(sysm: System) -> float:
    return sum(PSEUDO_ATOMS[t][3] for t in sysm.molecule.atom_types)


def _avg_err(values: Sequence[float]):
    v = np.asarray(values, float)
    n = len(v)
    s, s2 = v.sum(), (v * v).sum()
    return s / n, 2.0 * np.sqrt(abs(s2 / n - s * s / (n * n)))


def block_values(sysm: System, blocks: Sequence[Block]) -> Dict[str, List[float]]:
    """Per-block molecules per box, enthalpy of adsorption [K] and Widom
    weight (statistics.c:4077-4079 per block)."""
    n_mol, h_K, w = [], [], []
    for b in blocks:
        c = max(b.samples, 1.0)
        N, N2, U, UN = b.n / c, b.n2 / c, b.u / c, b.un / c
        var = N2 - N * N
        n_mol.append(N)
        h_K.append((UN - U * N) / var * units.ENERGY_TO_KELVIN - sysm.temperature if var > 0 else 0.0)
        w.append(b.widom_w / b.widom_n if b.widom_n > 0 else 0.0)
    return {"molecules": n_mol, "enthalpy_K": h_K, "widom_w": w}


def summary_text(sysm: System, blocks: Sequence[Block], title: Optional[str] = None) -> str:
    """The results sections of the reference's `.data` file for one
    system, from its block sums."""
    bv = block_values(sysm, blocks)
    name = sysm.molecule.name
    ncell = float(np.prod(sysm.unit_cells))
    fw_mass = framework_mass(sysm)
    volume = float(np.prod(sysm.box))
    to_mol_kg = 1000.0 * ncell / fw_mass
    to_mg_g = molecule_mass(sysm) * 1000.0 * ncell / fw_mass
    stp = units.MOLAR_GAS_CONSTANT * 273.15 / ATM_TO_PA
    to_cc_g = 1e6 * stp * ncell / fw_mass
    to_cc_cc = ncell * stp / (volume * units.ANGSTROM ** 3 * units.AVOGADRO_CONSTANT)
    out = []
    if title:
        out.append(title.rstrip("\n") + "\n\n")

    # enthalpy of adsorption
    out.append("Enthalpy of adsorption:\n=======================\n\n")
    for i, h in enumerate(bv["enthalpy_K"]):
        out.append("\tBlock[%2d] %-18.5f [K]\n" % (i, h))
    out.append(_LINE)
    h, he = _avg_err(bv["enthalpy_K"])
    kj = units.ENERGY_TO_KJ_PER_MOL / units.ENERGY_TO_KELVIN
    out.append("\tAverage   %18.5f +/- %18f [K]\n" % (h, he))
    out.append("\t          %18.5f +/- %18f [KJ/MOL]\n" % (h * kj, he * kj))
    out.append("\tNote: Ug should be subtracted from this value\n")
    out.append("\tNote: The heat of adsorption Q=-H\n\n\n")

    # number of molecules
    out.append("Number of molecules:\n====================\n\n")
    out.append("Component 0 [%s]\n" % name)
    out.append("-" * 61 + "\n")
    nm = bv["molecules"]
    avg, err = _avg_err(nm)
    for kind in ("absolute", "excess"):
        for i, v in enumerate(nm):
            out.append("\tBlock[%2d] %-18.5f [-]\n" % (i, v))
        out.append(_LINE)
        out.append("\tAverage                                %18.10f +/- %18.10f [-]\n" % (avg, err))
        out.append("\tAverage loading %s [molecules/unit cell]  %18.10f +/- %18.10f [-]\n"
                   % (kind, avg / ncell, err / ncell))
        for unit, f in (("mol/kg framework", to_mol_kg), ("milligram/gram framework", to_mg_g),
                        ("cm^3 (STP)/gr framework", to_cc_g), ("cm^3 (STP)/cm^3 framework", to_cc_cc)):
            out.append("\tAverage loading %s [%s]    %18.10f +/- %18.10f [-]\n"
                       % (kind, unit, avg * f / ncell, err * f / ncell))
        out.append("\n")
    out.append("\n")

    # Widom and Henry
    out.append("Average Widom Rosenbluth factor:\n================================\n")
    for i, v in enumerate(bv["widom_w"]):
        out.append("\tBlock[%2d] %-g [-]\n" % (i, v))
    out.append(_LINE)
    w, we = _avg_err(bv["widom_w"])
    out.append("\t[%s] Average Widom Rosenbluth-weight:   %g +/- %f [-]\n\n" % (name, w, we))
    # excess chemical potential -k_B T ln <W> [K] (statistics.c:4604-4625)
    mu = [-np.log(v) * sysm.temperature if v > 0 else 0.0 for v in bv["widom_w"]]
    out.append("Average Widom excess contribution:\n==================================\n")
    for i, v in enumerate(mu):
        out.append("\tBlock[%2d] %-g [-]\n" % (i, v))
    out.append(_LINE)
    m, me = _avg_err(mu)
    out.append("\t[%s] Average Widom excess chemical potential:   %g +/- %f [-]\n\n" % (name, m, me))
    density = 1e-3 * fw_mass / (volume * units.ANGSTROM ** 3 * units.AVOGADRO_CONSTANT)
    henry = [v / (sysm.ideal_gas_rosenbluth * units.MOLAR_GAS_CONSTANT * sysm.temperature * density)
             for v in bv["widom_w"]]
    out.append("Average Henry coefficient:\n==========================\n")
    for i, v in enumerate(henry):
        out.append("\tBlock[%2d] %-g [mol/kg/Pa]\n" % (i, v))
    out.append(_LINE)
    k, ke = _avg_err(henry)
    out.append("\t[%s] Average Henry coefficient:  %g +/- %g [mol/kg/Pa]\n\n" % (name, k, ke))
    # the next heading closes the Henry section for a parser that reads a
    # section up to the following rule, as the reference's output does
    out.append("Average adsorption energy <U_gh>_1-<U_h>_0 obtained from Widom-insertion:\n")
    out.append("(Note: the total heat of adsorption is dH=<U_gh>_1-<U_h>_0 - <U_g> - RT)\n")
    out.append("=" * 73 + "\n\n")
    out.append("Simulation finished,  0 warnings\n")
    return "".join(out)


_STATUS_LINE = re.compile(r"^\s*([A-Za-z/ \-]+?(?:energy|energy-drift)):\s+([-+\d.eE]+)")


def parse_energy_status(text: str, which: str = "initial full energy") -> Dict[str, float]:
    """Energies [K] of the block headed `Current (<which>) Energy Status`
    of a reference output file: {"Host/Adsorbate VDW energy": ..., ...}."""
    head = "Current (%s) Energy Status" % which
    i = text.find(head)
    if i < 0:
        raise KeyError(head)
    body = text[i + len(head):]
    j = body.find("Total energy:")
    body = body[: j + 200] if j >= 0 else body
    out: Dict[str, float] = {}
    for line in body.splitlines():
        m = _STATUS_LINE.match(line)
        if m:
            out[m.group(1).strip()] = float(m.group(2))
    m = re.search(r"Total energy:\s+([-+\d.eE]+)", body)
    if m:
        out["Total energy"] = float(m.group(1))
    return out
