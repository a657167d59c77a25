"""The oracle's Coulomb grid against the reference's (CPU): the real-space
Ewald derivatives of a unit probe charge at points
(CalculateDerivativesAtPositionReal), the grid file MakeGrid writes, and
InterpolateCoulombGrid for the charged CO2 sites
(tests/golden/grid_co2_coulomb.json)."""
import numpy as np
import pytest

from oracle import oracle as O
from raspa2_b200 import systems

from golden_cases import load, system_of


@pytest.fixture(scope="module")
def case():
    c = load("grid_co2_coulomb")
    s = system_of(c)
    o = O.Oracle.from_system(s)
    m = c["meta"]
    g = o.grid_build_coulomb(m["n"], m["size"], m["shift"])
    return c, s, o, g


def test_derivatives_match_reference(case):
    c, s, o, g = case
    for p, ref in zip(c["deriv_points"], c["deriv_ref"]):
        got = o.grid_derivatives_real(np.array(p))
        scale = np.abs(np.array(ref[:8])).max()
        np.testing.assert_allclose(got[:8], ref[:8], rtol=1e-9, atol=1e-12 * scale)
        assert abs(got[8] - ref[8]) <= 1e-12 * ref[8]


def test_grid_matches_reference_file(case):
    c, s, o, g = case
    flat = g.reshape(8, -1)
    got = flat[:, np.array(c["sample_index"])].T
    np.testing.assert_allclose(got, np.array(c["sample_values"]), rtol=2e-7, atol=1e-6)
    for m in range(8):
        ours = float(np.sum(flat[m].astype(np.float64)))
        assert abs(ours - c["plane_sums"][m]) <= 1e-6 * c["plane_abs_sums"][m] + 1e-6


def test_interpolation_matches_reference(case):
    """InterpolateCoulombGrid = charge x lookup; the grids agree to FP32
    rounding, so the bound is relative to the lookup's size."""
    c, s, o, g = case
    m = c["meta"]
    pts = np.array(c["interp_points"])
    got = []
    for name in c["types"]:
        q = systems.PSEUDO_ATOMS[name][2]
        got += [q * O.grid_interpolate(g, m["n"], m["size"], m["shift"], m["cell"], p) for p in pts]
    ref = np.array(c["interp_ref"])
    np.testing.assert_allclose(got, ref, rtol=2e-5, atol=1e-3)
