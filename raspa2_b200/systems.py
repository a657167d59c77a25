"""Seeded synthetic adsorption systems for the GCMC energy hot path.

A `System` holds everything the hot path needs: the rigid framework (positions,
pseudo-atom types, per-atom charges), the pseudo-atom table with its
Lennard-Jones parameters, the adsorbate molecule definitions, the cell, the
cut-off and the Ewald parameters, the state point and the MC move mix. The
same object is written out as RASPA input files (`raspa_io`) for the
reference and handed to the GPU engine, so both see the same numbers.

Frameworks are placed by seeded random sequential addition (Poisson-disk
sampling) under periodic boundaries with a minimum separation, as the
synthetic workloads prescribe; charges are drawn uniformly and shifted so
the framework is neutral.

Pseudo-atom names follow the RASPA force-field conventions
(`CH4_sp3`, `C_co2`, `O_co2`, `CH3_sp3`, `CH2_sp3`); the framework types are
named `Sifw` and `Ofw` so that no name is a prefix of another (the reference
matches pseudo-atom names by exact string, src/molecule.c:125-135).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

from . import units

# Lennard-Jones parameters (epsilon/k_B in K, sigma in Angstrom) and the
# default charge (e) of every pseudo-atom used by the synthetic workloads.
PSEUDO_ATOMS = {
    #  name       eps/K   sigma   charge  mass
    "Ofw":      (50.0,   3.00,   0.0,    15.9994),
    "Sifw":     (22.0,   2.30,   0.0,    28.0855),
    "CH4_sp3":  (148.0,  3.73,   0.0,    16.04246),
    "C_co2":    (27.0,   2.80,   0.70,   12.0),
    "O_co2":    (79.0,   3.05,  -0.35,   15.9994),
    "CH3_sp3":  (98.0,   3.75,   0.0,    15.03452),
    "CH2_sp3":  (46.0,   3.95,   0.0,    14.02658),
    # no interaction: the single atom of an otherwise empty box
    "Dummy":    (0.0,    1.00,   0.0,    1.0),
    # unit probe charge of the Coulomb grid (the reference's "UNIT", src/grids.c:637)
    "UNIT":     (0.0,    1.00,   1.0,    1.0),
}
TYPE_ORDER = list(PSEUDO_ATOMS.keys())


@dataclasses.dataclass
class Molecule:
    """An adsorbate: rigid (or single-bead), or a flexible linear chain.

    Rigid: `positions` is the reference geometry in Angstrom; `starting_bead`
    is the bead placed first by CBMC (src/cbmc.c:623 `HandleFirstBead`), the
    others are grown as one rigid group (src/cbmc.c:1480-1578).

    Flexible chain (rigid = False): atoms in chain order, grown from atom 0,
    fixed bond length `bond`, harmonic bends 0.5 k (theta - theta0)^2
    (`bend_k` in K/rad^2, `bend_theta0` in degrees) and TraPPE torsions
    (`torsion`, four coefficients in K), LJ between atoms four or more bonds
    apart; `positions` is then only a sample conformation.
    """
    name: str
    atom_types: List[str]
    positions: np.ndarray
    starting_bead: int = 0
    rigid: bool = True
    critical: tuple = (190.564, 4599200.0, 0.01142)
    bond: float = 0.0
    bend_k: float = 0.0
    bend_theta0: float = 0.0
    torsion: tuple = (0.0, 0.0, 0.0, 0.0)

    @property
    def n_atoms(self) -> int:
        return len(self.atom_types)

    def charges(self) -> np.ndarray:
        return np.array([PSEUDO_ATOMS[t][2] for t in self.atom_types], dtype=np.float64)


METHANE = Molecule("methane", ["CH4_sp3"], np.zeros((1, 3)), 0, True,
                   (190.564, 4599200.0, 0.01142))
CO2 = Molecule("CO2", ["O_co2", "C_co2", "O_co2"],
               np.array([[0.0, 0.0, 1.16], [0.0, 0.0, 0.0], [0.0, 0.0, -1.16]]),
               1, True, (304.1282, 7377300.0, 0.22394))


def _zigzag(n: int, bond: float, theta_deg: float) -> np.ndarray:
    """all-trans conformation of an n-bead chain"""
    th = np.deg2rad(theta_deg)
    dx, dy = bond * np.sin(th / 2.0), bond * np.cos(th / 2.0)
    return np.array([[i * dx, (i % 2) * dy, 0.0] for i in range(n)])


# united-atom n-hexane with TraPPE bends and torsions and 1.54 A bonds
HEXANE = Molecule("hexane", ["CH3_sp3"] + ["CH2_sp3"] * 4 + ["CH3_sp3"], _zigzag(6, 1.54, 114.0), 0, False,
                  (507.82, 3034000.0, 0.299), bond=1.54, bend_k=62500.0, bend_theta0=114.0,
                  torsion=(0.0, 355.03, -68.19, 791.32))


@dataclasses.dataclass
class MoveMix:
    """Relative move probabilities (normalised when used), in the engine's
    order: translation, rotation, CBMC insertion, CBMC deletion, CBMC
    reinsertion, Widom test insertion."""
    translation: float = 1.0
    rotation: float = 0.0
    swap_insert: float = 0.5   # a 'SwapProbability' p splits into p/2 insert + p/2 delete
    swap_delete: float = 0.5
    reinsertion: float = 0.0
    widom: float = 0.0

    def cumulative(self) -> np.ndarray:
        p = np.array([self.translation, self.rotation, self.swap_insert, self.swap_delete,
                      self.reinsertion, self.widom], float)
        return np.cumsum(p / p.sum())


@dataclasses.dataclass
class System:
    name: str
    unit_cell: np.ndarray            # (3,) cell lengths a, b, c, Angstrom
    unit_cells: np.ndarray           # (3,) replication
    frac: np.ndarray                 # (n_uc, 3) fractional positions in one unit cell
    uc_types: List[str]              # per unit-cell atom
    uc_charges: np.ndarray           # per unit-cell atom, e
    molecule: Molecule
    temperature: float
    pressure: float                  # Pa (fugacity, coefficient 1)
    cutoff: float = 12.0
    ewald: bool = False
    alpha: float = 0.265
    kmax: tuple = (8, 8, 8)
    trials: int = 10
    trials_first_bead: int = 10
    moves: MoveMix = dataclasses.field(default_factory=MoveMix)
    seed: int = 0
    max_translation: float = 1.0
    max_rotation_deg: float = 30.0
    # Rosenbluth weight of the molecule alone in an empty box (the
    # reference's IdealGasRosenbluthWeight); insertion and deletion
    # acceptance use W / ideal_gas_rosenbluth. 1 for rigid molecules.
    ideal_gas_rosenbluth: float = 1.0
    # bonded part of a flexible chain's CBMC trials: 0 = the reference's
    # scheme (src/cbmc.c:1580-2480: a shared bend angle per growth step,
    # `torsion_trials` torsion candidates per trial, the torsion Rosenbluth
    # factor in the weight), 1 = bend angle and dihedral drawn per trial
    chain_scheme: int = 0
    torsion_trials: int = 100          # NumberOfTrialPositionsTorsion
    # cell angles alpha, beta, gamma in degrees (the CIF's _cell_angle_*);
    # any angle other than 90 makes the box triclinic
    cell_angles: tuple = (90.0, 90.0, 90.0)

    # ----- derived quantities --------------------------------------------
    @property
    def box(self) -> np.ndarray:
        """box lengths along the cell vectors (a, b, c times the unit cells)"""
        return self.unit_cell * self.unit_cells

    @property
    def triclinic(self) -> bool:
        return any(float(x) != 90.0 for x in self.cell_angles)

    def _cell_matrix(self, lengths) -> np.ndarray:
        """Upper-triangular matrix whose columns are the cell vectors a, b, c
        for cell lengths `lengths` and the cell angles (src/framework.c:2003-2040)."""
        al, be, ga = (np.deg2rad(float(x)) for x in self.cell_angles)
        a, b, c = (float(x) for x in lengths)
        t = (np.cos(al) - np.cos(ga) * np.cos(be)) / np.sin(ga)
        return np.array([[a, b * np.cos(ga), c * np.cos(be)],
                         [0.0, b * np.sin(ga), c * t],
                         [0.0, 0.0, c * np.sqrt(1.0 - np.cos(be) ** 2 - t * t)]])

    @property
    def unit_cell_matrix(self) -> np.ndarray:
        if not self.triclinic:
            return np.diag(np.asarray(self.unit_cell, float))
        return self._cell_matrix(self.unit_cell)

    @property
    def box_matrix(self) -> np.ndarray:
        """cell vectors of the simulation box as columns"""
        if not self.triclinic:
            return np.diag(np.asarray(self.box, float))
        return self._cell_matrix(self.box)

    @property
    def volume(self) -> float:
        if not self.triclinic:
            return float(np.prod(self.box))
        return float(np.prod(np.diag(self.box_matrix)))

    def box_point(self, u) -> np.ndarray:
        """the point of fractional coordinates u (..., 3) in the box"""
        u = np.asarray(u, float)
        if not self.triclinic:
            return u * self.box
        return u @ self.box_matrix.T

    def min_image(self, d) -> np.ndarray:
        """minimum image of difference vectors d (..., 3): each fractional
        coordinate wrapped to the nearest integer (ApplyBoundaryCondition,
        src/potentials.h:232-268)"""
        d = np.asarray(d, float)
        if not self.triclinic:
            return d - self.box * np.rint(d / self.box)
        h = self.box_matrix
        s = d @ np.linalg.inv(h).T
        s -= np.rint(s)
        return s @ h.T

    def framework(self):
        """Cartesian framework atoms of the full simulation box.

        Returns (pos[N,3] float64, type[N] int32, charge[N] float64). Atoms are
        ordered like the reference builds its replicated cell: unit cells in
        x-major order, then the atoms of each cell in file order.
        """
        uc = self.unit_cell
        cells = []
        for i in range(int(self.unit_cells[0])):
            for j in range(int(self.unit_cells[1])):
                for k in range(int(self.unit_cells[2])):
                    cells.append((i, j, k))
        pos = []
        hu = self.unit_cell_matrix
        for (i, j, k) in cells:
            if self.triclinic:
                # the unit cell's atoms, shifted by whole cell vectors
                p = (self.frac + np.array([i, j, k], float)) @ hu.T
            else:
                p = np.empty_like(self.frac)
                p[:, 0] = uc[0] * self.frac[:, 0] + uc[0] * i
                p[:, 1] = uc[1] * self.frac[:, 1] + uc[1] * j
                p[:, 2] = uc[2] * self.frac[:, 2] + uc[2] * k
            pos.append(p)
        pos = np.concatenate(pos, axis=0) if pos else np.zeros((0, 3))
        ncell = len(cells)
        t = np.array([TYPE_ORDER.index(x) for x in self.uc_types] * ncell, dtype=np.int32)
        q = np.tile(self.uc_charges, ncell).astype(np.float64)
        return pos, t, q

    def n_framework(self) -> int:
        return len(self.uc_types) * int(np.prod(self.unit_cells))

    def lj_tables(self):
        """Lorentz-Berthelot mixed, truncated-and-shifted LJ table.

        Returns (eps[T,T] internal units, sigma2[T,T] A^2, shift[T,T]) where
        shift = U(rc) (src/potentials.c:5263-5287, 5867-5877).
        """
        n = len(TYPE_ORDER)
        eps = np.zeros((n, n))
        sig2 = np.zeros((n, n))
        shift = np.zeros((n, n))
        rc2 = self.cutoff ** 2
        for a, na in enumerate(TYPE_ORDER):
            for b, nb in enumerate(TYPE_ORDER):
                ea, sa = PSEUDO_ATOMS[na][:2]
                eb, sb = PSEUDO_ATOMS[nb][:2]
                e = math.sqrt(ea * eb) * units.KELVIN_TO_ENERGY
                s = 0.5 * (sa + sb)
                eps[a, b] = e
                sig2[a, b] = s * s
                r3 = (s * s / rc2) ** 3
                shift[a, b] = 4.0 * e * (r3 * (r3 - 1.0))
        return eps, sig2, shift

    def molecule_types(self) -> np.ndarray:
        return np.array([TYPE_ORDER.index(t) for t in self.molecule.atom_types], dtype=np.int32)

    def n_kvectors(self) -> int:
        return len(kvector_indices(self.kmax))


def kvector_indices(kmax: Sequence[int]) -> np.ndarray:
    """Integer wave vectors in the reference's order (src/ewald.c:532-599).

    kx runs 0..kmax_x (half space), ky and kz run -kmax..kmax; a vector is kept
    when 0 < kx^2+ky^2+kz^2 < (1.05*max(kmax))^2 (src/ewald.c:224-259).
    """
    kx, ky, kz = (int(k) for k in kmax)
    rc = (1.05 * max(kx, ky, kz)) ** 2
    out = []
    for i in range(0, kx + 1):
        for j in range(-ky, ky + 1):
            for k in range(-kz, kz + 1):
                s = i * i + j * j + k * k
                if s != 0 and s < rc:
                    out.append((i, j, k))
    return np.array(out, dtype=np.int32).reshape(-1, 3)


def pore_radius(cell: np.ndarray, void_fraction: float, rng: np.random.Generator) -> float:
    """Radius R of the cavity (points within R of the cell centre, minimum
    image) that leaves `void_fraction` of the cell empty."""
    s = rng.random((200000, 3)) - 0.5
    d = np.sqrt(np.sum((s * cell) ** 2, axis=1))
    return float(np.quantile(d, void_fraction))


def poisson_disk(rng: np.random.Generator, n: int, cell: np.ndarray, dmin: float,
                 pore: float = 0.0, max_rounds: int = 20000) -> np.ndarray:
    """Random sequential addition (Poisson-disk sampling) of `n` points in an
    orthorhombic periodic cell with minimum-image separation >= dmin.

    With pore > 0 the points are confined to the framework wall: outside the
    sphere of radius `pore` around the cell centre. Candidates are drawn in
    batches, screened against the accepted points with a periodic k-d tree
    and then accepted in draw order. Returns fractional coordinates."""
    from scipy.spatial import cKDTree

    cell = np.asarray(cell, float)
    pts = np.empty((0, 3))
    rounds = 0
    while len(pts) < n:
        rounds += 1
        if rounds > max_rounds:
            raise RuntimeError(f"poisson_disk: could not place {n} points (placed {len(pts)})")
        c = rng.random((256, 3))
        if pore > 0.0:
            d = (c - 0.5) * cell
            c = c[np.einsum("ij,ij->i", d, d) >= pore * pore]
        if len(pts):
            tree = cKDTree(np.mod(pts * cell, cell), boxsize=cell)
            dist, _ = tree.query(np.mod(c * cell, cell), k=1)
            c = c[dist >= dmin]
        for x in c:
            if len(pts) >= n:
                break
            if len(pts):
                d = pts - x
                d -= np.rint(d)
                d *= cell
                if np.min(np.einsum("ij,ij->i", d, d)) < dmin * dmin:
                    continue
            pts = np.vstack([pts, x[None, :]])
    return pts


def _quantise_frac(frac: np.ndarray) -> np.ndarray:
    # fractional coordinates are written with 12 decimals; keep exactly those
    return np.round(frac, 12)


def _neutral_charges(rng: np.random.Generator, n: int, qmax: float) -> np.ndarray:
    """Uniform charges in [-qmax, qmax], shifted to a neutral total.

    Charges are kept on a 1e-8 e lattice (the precision written to the CIF)
    and the lattice sum is made exactly zero, so the neutral framework the
    reference reads is the one the GPU sees."""
    q = rng.uniform(-qmax, qmax, n)
    q -= q.mean()
    iq = np.rint(q * 1e8).astype(np.int64)
    iq[-1] -= iq.sum()
    return iq.astype(np.float64) * 1e-8


def _assign_types(n: int, rng: np.random.Generator) -> List[str]:
    # one third Si, two thirds O, interleaved in a seeded random order
    n_si = n // 3
    labels = ["Sifw"] * n_si + ["Ofw"] * (n - n_si)
    perm = rng.permutation(n)
    return [labels[i] for i in perm]


# Share of the cell left empty by the framework wall. The workloads specify
# uniform Poisson-disk frameworks; at their densities (0.054 and 0.089
# atoms/A^3) a uniform layout leaves no cavity a molecule fits in (no
# insertion point with negative energy, Henry coefficient ~1e-6), so the
# sampling is confined to a wall around one cavity per unit cell.
VOID_FRACTION = 0.4


def methane_system(seed: int = 0, cycles_hint: int = 2000, layout: str = "porous") -> System:
    """Plain GCMC of single-site methane in a rigid neutral framework:
    orthorhombic 20.0 x 19.9 x 13.4 A cell replicated 2x2x3, 288 atoms per
    cell (96 Si, 192 O) at >= 1.6 A separation, 12 A truncated-shifted LJ,
    T = 300 K, fugacity 1e5 Pa, translation/insertion/deletion in equal
    proportion."""
    rng = np.random.default_rng(seed)
    cell = np.array([20.0, 19.9, 13.4])
    pore = pore_radius(cell, VOID_FRACTION, rng) if layout == "porous" else 0.0
    frac = _quantise_frac(poisson_disk(rng, 288, cell, 1.6, pore=pore))
    types = ["Sifw"] * 96 + ["Ofw"] * 192
    return System(
        name=f"methane_s{seed}", unit_cell=cell, unit_cells=np.array([2, 2, 3]),
        frac=frac, uc_types=types, uc_charges=np.zeros(288), molecule=METHANE,
        temperature=300.0, pressure=1e5, cutoff=12.0, ewald=False,
        moves=MoveMix(translation=1.0, rotation=0.0, swap_insert=0.5, swap_delete=0.5),
        seed=seed)


def methane_like_system(seed: int = 0, n_atoms: int = 288, temperature: float = 300.0,
                        pressure: float = 1e5) -> System:
    """Methane in a neutral Si/O framework of `n_atoms` atoms at the
    density of the 288-atom x 2x2x3 methane system (3456 atoms in
    40.0 x 39.8 x 40.2 A), in a cubic cell; cells narrower than 24 A are
    replicated 2x2x2."""
    rng = np.random.default_rng(seed)
    density = 3456.0 / (40.0 * 39.8 * 40.2)
    L = (n_atoms / density) ** (1.0 / 3.0)
    cell = np.array([L, L, L])
    pore = pore_radius(cell, VOID_FRACTION, rng)
    frac = _quantise_frac(poisson_disk(rng, n_atoms, cell, 1.6, pore=pore))
    n_si = n_atoms // 3
    types = ["Sifw"] * n_si + ["Ofw"] * (n_atoms - n_si)
    reps = np.array([2, 2, 2]) if L < 24.0 else np.array([1, 1, 1])
    return System(
        name=f"methane_n{n_atoms}_s{seed}", unit_cell=cell, unit_cells=reps,
        frac=frac, uc_types=types, uc_charges=np.zeros(n_atoms), molecule=METHANE,
        temperature=temperature, pressure=pressure, cutoff=12.0, ewald=False,
        moves=MoveMix(translation=1.0, rotation=0.0, swap_insert=0.5, swap_delete=0.5),
        seed=seed)


def torsion_rosenbluth(molecule: Molecule, temperature: float) -> float:
    """<exp(-U_torsion / k_B T)> over a uniform dihedral: the mean torsion
    Rosenbluth factor of one growth step of the reference's chain scheme."""
    phi = np.linspace(-np.pi, np.pi, 100001)[:-1]
    c = np.cos(phi)
    t = molecule.torsion
    u = t[0] + t[1] * (1 + c) + t[2] * (1 - np.cos(2 * phi)) + t[3] * (1 + np.cos(3 * phi))
    return float(np.mean(np.exp(-u / temperature)))


def chain_ideal_gas_estimate(molecule: Molecule, temperature: float) -> float:
    """Ideal-gas Rosenbluth weight of a linear chain under the reference's
    bonded scheme, without the intramolecular LJ (which raises n-hexane's by
    about 10 %): one torsion factor per bead from the fourth on. Runs whose
    averages depend on it measure it instead, by Widom insertions into an
    empty box (empty_box_system)."""
    return torsion_rosenbluth(molecule, temperature) ** max(molecule.n_atoms - 3, 0)


def hexane_system(seed: int = 4, n_atoms: int = 4096, cell: float = 40.0, temperature: float = 433.0,
                  pressure: float = 1e5, name: Optional[str] = None) -> System:
    """United-atom n-hexane (flexible chain, TraPPE bends and torsions, 1.54 A
    bonds) in a neutral Si/O framework of `n_atoms` atoms in a cubic cell,
    grown by CBMC with 8 first-bead trials and 16 trials per further bead, the
    bonded part as the reference draws it (100 torsion candidates per trial);
    translation, rotation, reinsertion and swap moves. The ideal-gas
    Rosenbluth weight is chain_ideal_gas_estimate's."""
    rng = np.random.default_rng(seed)
    c = np.array([cell, cell, cell], float)
    pore = pore_radius(c, VOID_FRACTION, rng)
    frac = _quantise_frac(poisson_disk(rng, n_atoms, c, 1.6, pore=pore))
    n_si = n_atoms // 3
    types = ["Sifw"] * n_si + ["Ofw"] * (n_atoms - n_si)
    reps = np.array([2, 2, 2]) if cell < 24.0 else np.array([1, 1, 1])
    return System(
        name=name or f"hexane_s{seed}", unit_cell=c, unit_cells=reps, frac=frac, uc_types=types,
        uc_charges=np.zeros(n_atoms), molecule=HEXANE, temperature=temperature, pressure=pressure,
        cutoff=12.0, ewald=False, trials=16, trials_first_bead=8,
        moves=MoveMix(translation=1.0, rotation=1.0, swap_insert=1.0, swap_delete=1.0, reinsertion=1.0),
        seed=seed, ideal_gas_rosenbluth=chain_ideal_gas_estimate(HEXANE, temperature))


def empty_box_system(molecule: Molecule, temperature: float, cell: float = 30.0, trials: int = 16,
                     trials_first_bead: int = 8) -> System:
    """`molecule` alone in an empty cubic box (one non-interacting framework
    atom), with Widom test insertions only: its average Rosenbluth weight is
    the ideal-gas Rosenbluth weight of the molecule for this CBMC scheme."""
    return System(
        name=f"empty_{molecule.name}", unit_cell=np.array([cell, cell, cell]), unit_cells=np.array([1, 1, 1]),
        frac=np.array([[0.5, 0.5, 0.5]]), uc_types=["Dummy"], uc_charges=np.zeros(1), molecule=molecule,
        temperature=temperature, pressure=1e5, cutoff=12.0, ewald=False, trials=trials,
        trials_first_bead=trials_first_bead,
        moves=MoveMix(translation=0.0, rotation=0.0, swap_insert=0.0, swap_delete=0.0, widom=1.0), seed=0)


def co2_system(seed: int = 1, n_atoms: int = 1536, cell: float = 25.8,
               kmax: int = 8, temperature: float = 298.0, pressure: float = 1e5,
               dmin: float = 1.5, name: Optional[str] = None, layout: str = "porous") -> System:
    """Rigid 3-site CO2 in a charged cubic framework: `n_atoms` atoms placed
    at >= `dmin` separation, charges uniform in [-1.2, 1.2] e shifted to net
    zero, Ewald alpha = 0.265/A with kmax per axis, 12 A cut-off, CBMC
    insertion/deletion with 10 first-bead trials x 10 orientations,
    translation and rotation. Cells narrower than 24 A are replicated 2x2x2,
    as the reference requires a box of at least twice the cut-off."""
    rng = np.random.default_rng(seed)
    c = np.array([cell, cell, cell], float)
    pore = pore_radius(c, VOID_FRACTION, rng) if layout == "porous" else 0.0
    frac = _quantise_frac(poisson_disk(rng, n_atoms, c, dmin, pore=pore))
    types = _assign_types(n_atoms, rng)
    q = _neutral_charges(rng, n_atoms, 1.2)
    reps = np.array([2, 2, 2]) if cell < 24.0 else np.array([1, 1, 1])
    return System(
        name=name or f"co2_s{seed}", unit_cell=c, unit_cells=reps, frac=frac,
        uc_types=types, uc_charges=q, molecule=CO2, temperature=temperature,
        pressure=pressure, cutoff=12.0, ewald=True, alpha=0.265,
        kmax=(kmax, kmax, kmax), trials=10, trials_first_bead=10,
        moves=MoveMix(translation=1.0, rotation=1.0, swap_insert=1.0, swap_delete=1.0),
        seed=seed)


def co2_triclinic_system(seed: int = 11, n_atoms: int = 2000, cell=(29.0, 28.0, 30.0),
                         angles=(80.0, 95.0, 110.0)) -> System:
    """The CO2 model of co2_system in a triclinic cell: lengths `cell`,
    angles alpha, beta, gamma = `angles` (perpendicular widths 27.2, 26.0 and
    29.5 A, so one cell holds the 12 A cut-off sphere). The framework's
    fractional positions are a Poisson-disk set drawn in a cube of the same
    density, then taken as fractions of the triclinic cell."""
    base = co2_system(seed=seed, n_atoms=n_atoms, cell=float((n_atoms / 0.0894) ** (1.0 / 3.0)),
                      name=f"co2tri_s{seed}")
    return dataclasses.replace(base, unit_cell=np.array(cell, float), unit_cells=np.array([1, 1, 1]),
                               cell_angles=tuple(float(x) for x in angles))


def batched_co2_systems(n: int = 64, seed: int = 2) -> List[System]:
    """Independent CO2 systems of uneven size: cubic cells 18-36 A with
    512-4096 framework atoms (framework density held near the 1536-atom /
    25.8 A reference), kmax 6-10 per axis, pressures log-spaced 1e3-1e7 Pa,
    T in {273, 298, 323} K, each seeded on its own."""
    rng = np.random.default_rng(seed)
    out = []
    pressures = np.logspace(3, 7, n)
    temps = (273.0, 298.0, 323.0)
    for i in range(n):
        cell = float(rng.uniform(18.0, 36.0))
        natoms = int(np.clip(round(1536 * (cell / 25.8) ** 3), 512, 4096))
        kmax = int(rng.integers(6, 11))
        out.append(co2_system(seed=seed * 1000 + i, n_atoms=natoms, cell=cell, kmax=kmax,
                              temperature=temps[i % 3], pressure=float(pressures[i]),
                              name=f"co2_b{i}"))
    return out


def tiny_co2_system(seed: int = 7, n_atoms: int = 96, cell: float = 24.5,
                    kmax: int = 3) -> System:
    """A small charged system for fast exact checks (a few hundred atoms)."""
    return co2_system(seed=seed, n_atoms=n_atoms, cell=cell, kmax=kmax, dmin=1.5,
                      name=f"co2tiny_s{seed}")
