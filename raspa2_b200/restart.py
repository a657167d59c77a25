"""Text restart files in the reference's schema.

The reference writes one restart file per system at every `PrintEvery`
cycle and at the end of a run (PrintRestartFile, src/output.c:7296-7700,
called from src/monte_carlo.c:179,618,1044) and reads it back when the
input says `RestartFile yes` (ReadRestartFile, src/input.c:8524-9000, from
`RestartInitial/System_<n>/`). A file written here is read by the reference,
and a file the reference wrote is read here, so a configuration moves
between the two codes in either direction:

- `write_restart` writes the cell block, the MC maximum changes, the
  component block and the adsorbate records (positions; zero velocities and
  forces; charges, scaling 1, not fixed) exactly as the reference lays them
  out;
- `read_restart` parses the records the hot path needs: cells, maximum
  translation and rotation per component, and the molecule positions per
  component (`Adsorbate-atom-position: molecule atom x y z`).

Only adsorbates are handled (no cations, no fractional molecules, no
reactions), as in the rest of this package.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional

import numpy as np

from .systems import System

_RULE = "=" * 72 + "\n"


def restart_file_name(sysm: System) -> str:
    """`restart_<framework>_<a>.<b>.<c>_<T>_<P>` (src/output.c:7320-7328;
    the temperature as %lf, the pressure in Pa as %lg)."""
    a, b, c = (int(x) for x in sysm.unit_cells)
    return "restart_%s_%d.%d.%d_%f_%g" % (sysm.name, a, b, c, float(sysm.temperature), float(sysm.pressure))


def restart_path(sysm: System, directory: str, system_index: int = 0, initial: bool = True) -> str:
    """Where the reference looks for (RestartInitial/) or writes (Restart/)
    the restart file of system `system_index`."""
    sub = "RestartInitial" if initial else "Restart"
    return os.path.join(directory, sub, f"System_{system_index}", restart_file_name(sysm))


def write_restart(path: str, sysm: System, xyz: np.ndarray, max_translation: Optional[float] = None,
                  max_rotation: Optional[float] = None) -> str:
    """Writes molecule positions `xyz` [n_mol, n_atom, 3] of the one
    adsorbate component of `sysm` as a restart file the reference reads
    (maximum translation in A, maximum rotation in radians)."""
    xyz = np.asarray(xyz, float).reshape(-1, sysm.molecule.n_atoms, 3)
    mt = sysm.max_translation if max_translation is None else max_translation
    mr = np.deg2rad(sysm.max_rotation_deg) if max_rotation is None else max_rotation   # radians
    uc, box = sysm.unit_cell, sysm.box
    lines = ["Cell info:\n", _RULE]
    lines.append("number-of-unit-cells: %d %d %d\n" % tuple(int(x) for x in sysm.unit_cells))
    for name, vec in zip("abc", np.diag(uc)):
        lines.append("unit-cell-vector-%s: %18.12f %18.12f %18.12f\n" % (name, *vec))
    lines.append("\n")
    for name, vec in zip("abc", np.diag(box)):
        lines.append("cell-vector-%s: %18.12f %18.12f %18.12f\n" % (name, *vec))
    lines.append("\n")
    lines.append("cell-lengths: %18.12f %18.12f %18.12f\n" % tuple(uc))
    lines.append("cell-angles: %18.12f %18.12f %18.12f\n" % (90.0, 90.0, 90.0))
    lines.append("\n\n")
    lines += ["Maximum changes for MC-moves:\n", _RULE]
    lines.append("Maximum-volume-change: %f\n" % 0.001563)
    lines.append("Maximum-Gibbs-volume-change: %f\n" % 0.00625)
    lines.append("Maximum-box-shape-change: " + ", ".join(["%f %f %f" % (0.1, 0.1, 0.1)] * 3) + "\n")
    lines.append("\n\n")
    lines += ["Acceptance targets for MC-moves:\n", _RULE]
    lines.append("Target-volume-change: %f\n" % 0.5)
    lines.append("Target-box-shape-change: %f\n" % 0.5)
    lines.append("Target-Gibbs-volume-change: %f\n" % 0.5)
    lines.append("\n\n")
    m = sysm.molecule
    lines.append("Components: 1 (Adsorbates %d, Cations 0)\n" % len(xyz))
    lines.append(_RULE)
    lines.append("Component 0 (%s)\n" % m.name)
    lines.append("\tFractional-molecule-id component 0: -1\n")
    lines.append("\tLambda-factors component 0: " + " ".join(["%f" % 0.0] * m.n_atoms) + "\n")
    lines.append("\tNumber-of-biasing-factors component 0: 21\n")
    lines.append("\tBiasing-factors component 0: " + " ".join(["%f" % 0.0] * 21) + "\n")
    lines.append("\tMaximum-CF-Lambda-change component 0: %f\n" % 0.5)
    lines.append("\tMaximum-CBCF-Lambda-change component 0: %f\n" % 0.5)
    lines.append("\n")
    lines.append("\tMaximum-translation-change component 0: %f,%f,%f\n" % (mt, mt, mt))
    lines.append("\tMaximum-translation-in-plane-change component 0: %f,%f,%f\n" % (0.0, 0.0, 0.0))
    lines.append("\tMaximum-rotation-change component 0: %f %f %f\n" % (mr, mr, mr))
    lines.append("\n")
    lines.append("Reactions: 0\n")
    lines.append("\n")
    lines.append("Component: %d     %s    %d molecules of %s\n" % (0, "Adsorbate", len(xyz), m.name))
    lines.append("-" * 72 + "\n")
    q = m.charges()
    for k, mol in enumerate(xyz):
        for a, p in enumerate(mol):
            lines.append("Adsorbate-atom-position: %d %d %18.12f %18.12f %18.12f\n" % (k, a, *p))
    for rec in ("velocity", "force"):
        pad = " " * (len("position") - len(rec))
        for k in range(len(xyz)):
            for a in range(m.n_atoms):
                lines.append("Adsorbate-atom-%s:%s %d %d %18.12f %18.12f %18.12f\n" % (rec, pad, k, a, 0.0, 0.0, 0.0))
    for k in range(len(xyz)):
        for a in range(m.n_atoms):
            lines.append("Adsorbate-atom-charge:   %d %d %18.12f\n" % (k, a, q[a]))
    for k in range(len(xyz)):
        for a in range(m.n_atoms):
            lines.append("Adsorbate-atom-scaling:  %d %d %18.12f\n" % (k, a, 1.0))
    for k in range(len(xyz)):
        for a in range(m.n_atoms):
            lines.append("Adsorbate-atom-fixed:    %d %d       %d %d %d\n" % (k, a, 0, 0, 0))
    lines.append("\n\n")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w") as fh:
        fh.writelines(lines)
    return path


@dataclasses.dataclass
class RestartComponent:
    name: str
    positions: np.ndarray                     # [n_mol, n_atom, 3]
    max_translation: Optional[np.ndarray] = None
    max_rotation: Optional[np.ndarray] = None


@dataclasses.dataclass
class Restart:
    unit_cells: np.ndarray                    # (3,) replication
    unit_cell_vectors: np.ndarray             # (3, 3) rows a, b, c
    cell_vectors: np.ndarray                  # (3, 3) of the simulation box
    components: List[RestartComponent]

    def component(self, name: str) -> RestartComponent:
        for c in self.components:
            if c.name == name:
                return c
        raise KeyError(name)


def read_restart(path: str) -> Restart:
    """Parses a restart file of the reference (or of `write_restart`)."""
    unit_cells = np.ones(3, int)
    ucv = np.zeros((3, 3))
    cv = np.zeros((3, 3))
    names: Dict[int, str] = {}
    mt: Dict[int, np.ndarray] = {}
    mr: Dict[int, np.ndarray] = {}
    counts: Dict[int, int] = {}
    order: List[int] = []          # component of each "Component:" block, in file order
    pos: Dict[int, Dict[int, Dict[int, np.ndarray]]] = {}
    current = None
    with open(path) as fh:
        for raw in fh:
            line = raw.strip()
            if not line:
                continue
            key, _, rest = line.partition(" ")
            rest = rest.strip()
            if key == "number-of-unit-cells:":
                unit_cells = np.array([int(x) for x in rest.split()[:3]])
            elif key.startswith("unit-cell-vector-"):
                ucv["abc".index(key[-2])] = [float(x) for x in rest.split()[:3]]
            elif key.startswith("cell-vector-"):
                cv["abc".index(key[-2])] = [float(x) for x in rest.split()[:3]]
            elif key == "Component" and "(" in rest:
                idx = int(rest.split()[0])
                names[idx] = rest[rest.index("(") + 1: rest.rindex(")")]
            elif key == "Maximum-translation-change" and rest.startswith("component"):
                idx = int(rest.split()[1].rstrip(":"))
                mt[idx] = np.array([float(x) for x in rest.split(":", 1)[1].replace(",", " ").split()])
            elif key == "Maximum-rotation-change" and rest.startswith("component"):
                idx = int(rest.split()[1].rstrip(":"))
                mr[idx] = np.array([float(x) for x in rest.split(":", 1)[1].split()])
            elif key == "Component:":
                f = rest.split()
                current = int(f[0])
                counts[current] = int(f[2])
                order.append(current)
                pos.setdefault(current, {})
            elif key == "Adsorbate-atom-position:":
                if current is None:
                    raise ValueError(f"{path}: adsorbate record before its component block")
                f = rest.split()
                k, a = int(f[0]), int(f[1])
                pos[current].setdefault(k, {})[a] = np.array([float(x) for x in f[2:5]])
    comps = []
    for idx in sorted(names):
        mols = pos.get(idx, {})
        n = counts.get(idx, 0)
        if len(mols) != n:
            raise ValueError(f"{path}: component {idx} declares {n} molecules, holds {len(mols)}")
        if n:
            na = len(mols[min(mols)])
            arr = np.array([[mols[k][a] for a in range(na)] for k in sorted(mols)])
        else:
            arr = np.zeros((0, 0, 3))
        comps.append(RestartComponent(names[idx], arr, mt.get(idx), mr.get(idx)))
    return Restart(unit_cells, ucv, cv, comps)
