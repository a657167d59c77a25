"""Energy grids of a triclinic cell (the co2_triclinic system: angles 80, 95,
110 degrees): the oracle's MakeGrid and its lookup, wrapped into the unit
cell through fractional coordinates, against the reference's grid files and
its InterpolateVDWGrid / InterpolateCoulombGrid (their TRICLINIC branches,
src/grids.c:1004-1021) in tests/golden/grid_co2_triclinic.json."""
import numpy as np
import pytest

from oracle import oracle as O
from raspa2_b200 import systems

from golden_cases import load, system_of


@pytest.fixture(scope="module")
def case():
    c = load("grid_co2_triclinic")
    s = system_of(c)
    o = O.Oracle.from_system(s)
    grids = {}
    for k, m in c["meta"].items():
        if k == "coulomb":
            grids[k] = o.grid_build_coulomb(m["n"], m["size"], m["shift"])
        else:
            grids[k] = o.grid_build(systems.TYPE_ORDER.index(k), m["n"], m["size"], m["shift"])
    return c, s, o, grids


@pytest.mark.parametrize("kind", ["C_co2", "O_co2", "coulomb"])
def test_grid_matches_reference_file(case, kind):
    c, s, o, grids = case
    flat = grids[kind].reshape(8, -1)
    smp = c["samples"][kind]
    got = flat[:, np.array(smp["index"])].T
    np.testing.assert_allclose(got, np.array(smp["values"]), rtol=2e-7, atol=1e-6)
    ps = c["plane_sums"][kind]
    for m in range(8):
        ours = float(np.sum(flat[m].astype(np.float64)))
        assert abs(ours - ps["sum"][m]) <= 1e-6 * ps["abs"][m] + 1e-6


def test_lookups_match_reference(case):
    """The lookups on the oracle's grids (equal to the reference's to FP32
    rounding), with the point wrapped into the triclinic unit cell, equal the
    reference's on its own files."""
    c, s, o, grids = case
    ucm = s.unit_cell_matrix
    pts = np.array(c["points"])
    for name in c["types"]:
        m = c["meta"][name]
        got = [O.grid_interpolate(grids[name], m["n"], m["size"], m["shift"], m["cell"], p, cell_matrix=ucm)
               for p in pts]
        np.testing.assert_allclose(got, c["interp_ref"][name]["vdw"], rtol=2e-5, atol=1e-3)
        mc = c["meta"]["coulomb"]
        q = systems.PSEUDO_ATOMS[name][2]
        got = [q * O.grid_interpolate(grids["coulomb"], mc["n"], mc["size"], mc["shift"], mc["cell"], p,
                                      cell_matrix=ucm) for p in pts]
        np.testing.assert_allclose(got, c["interp_ref"][name]["coulomb"], rtol=2e-5, atol=1e-3)
