"""Pins the C oracle (oracle/oracle.c) to the reference's own outputs.

The fixtures in tests/golden/ were produced by the reference's energy, Ewald,
CBMC and grid routines (tests/golden/make_golden.py). Everything here runs on
the CPU.
"""
import numpy as np
import pytest

from oracle import oracle as O
from raspa2_b200 import systems, units

from golden_cases import ENERGY_CASES, load, system_of

RTOL = 1e-10


def close(a, b, rtol=RTOL, atol=1e-9):
    np.testing.assert_allclose(np.asarray(a, float), np.asarray(b, float), rtol=rtol, atol=atol)


@pytest.fixture(scope="module", params=ENERGY_CASES)
def case(request):
    c = load(request.param)
    s = system_of(c)
    o = O.Oracle.from_system(s)
    o.set_molecules(np.array(c["molecules"]))
    return c, s, o


def test_system_matches_reference_input(case):
    c, s, o = case
    # the generator's framework is the one the reference read from the CIF
    assert c["framework_max_abs_diff_vs_generator"] < 1e-12
    assert c["n_framework"] == s.n_framework()
    # pseudo-atom table: the reference prepends UNIT, then the file order
    # the fixture's pseudo-atom order (after the reference's UNIT) is a
    # prefix of ours: types added later keep every earlier index
    names = c["pseudo_names"][1:]
    assert systems.TYPE_ORDER[:len(names)] == names
    const = c["constants"]
    close(const[0], units.COULOMBIC_CONVERSION_FACTOR, rtol=1e-15)
    close(const[1], units.KELVIN_TO_ENERGY, rtol=1e-15)
    close(const[4], units.beta(s.temperature), rtol=1e-15)
    assert const[5] == units.ENERGY_OVERLAP_CRITERIA
    if s.ewald:
        assert int(c["ewald"][4]) == s.n_kvectors()
        close(c["ewald"][0], s.alpha, rtol=1e-15)
        # UIon of the reference (EwaldEnergyIon)
        close(o.s.uion, c["ewald"][6], rtol=1e-12)


def test_total_energy(case):
    c, s, o = case
    close(o.total_energy(), c["energy"][0][:6])


def test_bead_energies_at_points(case):
    c, s, o = case
    q = s.molecule.charges()
    t = s.molecule_types()
    for pt in c["points"]:
        a = pt["atom"]
        ours = o.point(int(t[a]), float(q[a]), np.array(pt["p"]), exclude=pt["exclude"])
        close(ours, pt["ref"])


def test_move_differences(case):
    c, s, o = case
    n_overlap = 0
    for mv in c["moves"]:
        ov, dl = o.move_delta(mv["m"], np.array(mv["new"]))
        ref = mv["ref"]
        assert bool(ref[0]) == ov
        if ov:
            n_overlap += 1
            continue
        close(dl, ref[1:5])
        if s.ewald:
            de, _ = o.ewald_delta(old=o.molecules()[mv["m"]], new=np.array(mv["new"]))
            close([de[1], de[0]], ref[5:7], atol=1e-8)
    assert n_overlap >= 1          # the fixture includes an overlapping move


def test_fourier_insert_delete(case):
    c, s, o = case
    if not s.ewald:
        pytest.skip("no charges")
    de, _ = o.ewald_delta(new=np.array(c["insert"]))
    close([de[1], de[0], de[2]], c["fourier"][0][5:8], atol=1e-8)
    m = len(c["molecules"]) - 1
    de, _ = o.ewald_delta(old=o.molecules()[m])
    close([de[1], de[0], de[2]], c["fourier"][1][5:8], atol=1e-8)


def test_accepted_move_then_dependent_move(case):
    """S(k) bookkeeping across an accepted move (AcceptEwaldAdsorbateMove)."""
    c, s, o0 = case
    if not c["accepted"]:
        pytest.skip("needs two molecules")
    o = O.Oracle.from_system(s)
    o.set_molecules(np.array(c["molecules"]))
    a, b = c["accepted"]
    ov, dl = o.move_delta(a["m"], np.array(a["new"]))
    assert not ov
    de, sk = o.ewald_delta(old=o.molecules()[a["m"]], new=np.array(a["new"]))
    close(dl, c["accepted_ref"][0][1:5])
    # accept: positions and S(k) from the candidate
    o.ads[a["m"]] = np.array(a["new"])
    if s.ewald:
        o.sk_ads[:] = sk[: o.s.nk]
    ov, dl = o.move_delta(b["m"], np.array(b["new"]))
    close(dl, c["accepted_ref"][1][1:5])
    if s.ewald:
        de, _ = o.ewald_delta(old=o.molecules()[b["m"]], new=np.array(b["new"]))
        close([de[1], de[0]], c["accepted_ref"][1][5:7], atol=1e-8)
    close(o.total_energy(), c["energy"][1][:6])


def test_cbmc_with_reference_random_stream(case):
    """CBMC growth/retrace driven by the reference's MT19937-64 stream gives
    the reference's Rosenbluth weights, energies, grown positions and the same
    number of random draws (the next draw matches)."""
    c, s, o0 = case
    o = O.Oracle.from_system(s)
    mols = np.array(c["molecules"])
    for acc in c["accepted"][:1]:
        mols[acc["m"]] = np.array(acc["new"])
    o.set_molecules(mols)
    nf, nt = c["trials"]
    na = s.molecule.n_atoms
    for cb in c["cbmc"]:
        ref = cb["ref"]
        if cb["kind"] == "insert":
            out, nx, nxt = o.cbmc_insert_mt(cb["seed"], nf, nt)
            assert bool(ref[0]) == bool(out[0])
            if not out[0]:
                close(out[1], ref[1], rtol=1e-9, atol=0)
                close(out[2:6], ref[2:6])
                close(nx.reshape(-1), ref[6:6 + 3 * na])
            close(nxt, ref[-1], rtol=0, atol=0)
        else:
            out, nxt = o.cbmc_delete_mt(cb["m"], cb["seed"], nf, nt)
            assert bool(ref[0]) == bool(out[0])
            if not out[0]:
                close(out[1], ref[1], rtol=1e-9, atol=0)
                close(out[2:6], ref[2:6])
            close(nxt, ref[-1], rtol=0, atol=0)


@pytest.fixture(scope="module")
def grid_case():
    c = load("grid_methane")
    s = system_of(c)
    o = O.Oracle.from_system(s)
    return c, s, o


def test_grid_derivatives(grid_case):
    c, s, o = grid_case
    t = systems.TYPE_ORDER.index("CH4_sp3")
    for p, ref in zip(c["deriv_points"], c["deriv_ref"]):
        close(o.grid_derivatives(t, np.array(p)), ref, rtol=1e-10, atol=1e-7)


def test_grid_build_matches_reference_file(grid_case):
    c, s, o = grid_case
    m = c["meta"]
    t = systems.TYPE_ORDER.index("CH4_sp3")
    g = o.grid_build(t, m["n"], m["size"], m["shift"])
    flat = g.reshape(8, -1)
    got = flat[:, np.array(c["sample_index"])].T
    np.testing.assert_allclose(got, np.array(c["sample_values"]), rtol=2e-7, atol=1e-6)
    sums = [float(np.sum(flat[k].astype(np.float64))) for k in range(8)]
    np.testing.assert_allclose(sums, c["plane_sums"], rtol=1e-6)


def test_grid_interpolation_matches_reference(grid_case):
    """InterpolateVDWGrid (Lekien-Marsden matrix form) equals the tensor-product
    Hermite evaluation on the same grid."""
    c, s, o = grid_case
    m = c["meta"]
    t = systems.TYPE_ORDER.index("CH4_sp3")
    g = o.grid_build(t, m["n"], m["size"], m["shift"])
    for p, ref in zip(c["interp_points"], c["interp_ref"]):
        v = O.grid_interpolate(g, m["n"], m["size"], m["shift"], m["cell"], np.array(p))
        close(v, ref, rtol=1e-7, atol=1e-6)


def test_philox_known_answer():
    """Philox4x32-10 known-answer vectors of the published reference
    implementation (Random123 kat_vectors): counter/key all zero and all ones."""
    import ctypes as C
    L = O.lib()
    out = (C.c_uint32 * 4)()
    ctr = (C.c_uint32 * 4)(0, 0, 0, 0)
    key = (C.c_uint32 * 2)(0, 0)
    L.or_philox4x32(ctr, key, out)
    assert list(out) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    ctr = (C.c_uint32 * 4)(0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF)
    key = (C.c_uint32 * 2)(0xFFFFFFFF, 0xFFFFFFFF)
    L.or_philox4x32(ctr, key, out)
    assert list(out) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
