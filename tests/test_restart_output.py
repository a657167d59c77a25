"""Restart files and results in the reference's formats (CPU).

- A restart file the reference wrote (tests/golden/restart_*.txt, made by
  tests/golden/make_restart_golden.py) is read here, and the oracle's
  energies of those molecules equal the energies the reference printed for
  the same configuration.
- A restart file written here is read back unchanged, and the reference
  program reads it (`RestartFile yes`) and prints the oracle's energies for
  it (skipped when the reference program has not been built).
- The `.data` summary written here is read by the reference's own output
  parser (skipped when the reference's sources are absent).
"""
import dataclasses
import glob
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import REFROOT
from oracle import oracle as O
from raspa2_b200 import output, raspa_io, restart, systems, units

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
ROOT = os.path.dirname(HERE)
SIMULATE = os.path.join(ROOT, "oracle", "_ref", "simulate")
REF_PYTHON = os.path.join(REFROOT, "python")

CASES = {
    "co2_config1": lambda: systems.co2_system(seed=1),
    "hexane_small": lambda: systems.hexane_system(seed=4, n_atoms=1200, cell=26.0),
}


def case_system(name):
    meta = json.load(open(os.path.join(GOLDEN, f"restart_{name}.json")))
    s = dataclasses.replace(CASES[name](), pressure=meta["pressure_Pa"], temperature=meta["temperature_K"])
    return s, meta


def oracle_energies_K(s, xyz):
    """The reference's energy-status entries, from the oracle, in K."""
    o = O.Oracle.from_system(s, maxmol=max(len(xyz), 1))
    o.set_molecules(xyz)
    u = o.total_energy() * units.ENERGY_TO_KELVIN
    e = {"Host/Adsorbate VDW energy": u[0], "Adsorbate/Adsorbate VDW energy": u[1],
         "Host/Adsorbate charge-charge Real energy": u[2], "Adsorbate/Adsorbate charge-charge Real energy": u[3],
         "Host/Adsorbate charge-charge Fourier energy": u[4],
         "Adsorbate/Adsorbate charge-charge Fourier energy": u[5]}
    if not s.molecule.rigid:
        e["intra"] = o.intra_energy() * units.ENERGY_TO_KELVIN
    return e


def assert_energies_match(ours, ref):
    for k, v in ours.items():
        if k == "intra":
            r = ref["Adsorbate bend energy"] + ref["Adsorbate torsion energy"] + ref["Adsorbate intra VDW energy"]
        else:
            r = ref[k]
        # the reference prints 8 decimals
        assert abs(v - r) <= 1e-9 * abs(r) + 2e-8, (k, v, r)


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_restart_file_gives_reference_energies(name):
    s, meta = case_system(name)
    r = restart.read_restart(os.path.join(GOLDEN, f"restart_{name}.txt"))
    assert r.unit_cells.tolist() == [int(x) for x in s.unit_cells]
    np.testing.assert_allclose(np.diag(r.cell_vectors), s.box, rtol=0, atol=1e-9)
    c = r.component(s.molecule.name)
    assert c.positions.shape[1:] == (s.molecule.n_atoms, 3) and len(c.positions) > 0
    assert restart.restart_file_name(s) == meta["restart_file_name"]
    assert_energies_match(oracle_energies_K(s, c.positions), meta["energies_K"])


def test_write_read_round_trip(tmp_path):
    s, _ = case_system("co2_config1")
    xyz = restart.read_restart(os.path.join(GOLDEN, "restart_co2_config1.txt")).components[0].positions
    p = restart.write_restart(restart.restart_path(s, str(tmp_path)), s, xyz, max_translation=0.7, max_rotation=0.3)
    r = restart.read_restart(p)
    np.testing.assert_allclose(r.components[0].positions, xyz, rtol=0, atol=1e-12)
    np.testing.assert_allclose(r.components[0].max_translation, [0.7] * 3)
    np.testing.assert_allclose(r.components[0].max_rotation, [0.3] * 3)
    assert r.components[0].name == s.molecule.name


@pytest.mark.skipif(not os.path.exists(SIMULATE), reason="reference program not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_reads_our_restart_file(tmp_path, name):
    """Molecules moved by the oracle's MC, written here, read by the
    reference: its initial full energies equal the oracle's."""
    s, _ = case_system(name)
    xyz = restart.read_restart(os.path.join(GOLDEN, f"restart_{name}.txt")).components[0].positions
    o = O.Oracle.from_system(s, maxmol=len(xyz) + 16)
    o.set_molecules(xyz)
    st = O.MCState()
    o.mc_run(O.mc_params(dataclasses.replace(s, moves=systems.MoveMix(translation=1.0, rotation=1.0,
                                                                     swap_insert=0.0, swap_delete=0.0)),
                         5, 0), st, 0, 200)
    moved = o.molecules()
    assert np.abs(moved - xyz).max() > 0.1
    d = str(tmp_path)
    raspa_io.write_inputs(s, d, cycles=0, init_cycles=0, print_every=10 ** 9, seed=1, restart=True)
    restart.write_restart(restart.restart_path(s, d), s, moved)
    r = subprocess.run([SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-500:]
    data = glob.glob(os.path.join(d, "Output", "System_0", "*.data"))[0]
    txt = open(data).read()
    ref = output.parse_energy_status(txt, "initial full energy")
    assert_energies_match(oracle_energies_K(s, moved), ref)


def _blocks():
    rng = np.random.default_rng(3)
    out = []
    for _ in range(5):
        n = 1000.0
        N = 2.7 + 0.1 * rng.random()
        out.append(output.Block(n, N * n, (N * N + 0.4) * n, -900.0 * n, -900.0 * N * n - 300.0 * n, 2.0, 1000.0))
    return out


def test_summary_numbers():
    s, _ = case_system("hexane_small")
    bl = _blocks()
    bv = output.block_values(s, bl)
    txt = output.summary_text(s, bl)
    avg = np.mean(bv["molecules"])
    assert "Average loading absolute [molecules/unit cell]  %18.10f" % avg in txt
    # enthalpy per block: cov(U, N) / var(N) - k_B T, in K
    b = bl[0]
    N, N2, U, UN = b.n / b.samples, b.n2 / b.samples, b.u / b.samples, b.un / b.samples
    h = ((UN - U * N) / (N2 - N * N)) * units.ENERGY_TO_KELVIN - s.temperature
    assert abs(bv["enthalpy_K"][0] - h) < 1e-9 * abs(h)


@pytest.mark.skipif(not os.path.isdir(REF_PYTHON), reason="reference sources absent")
def test_reference_parser_reads_our_summary():
    sys.path.insert(0, REF_PYTHON)
    try:
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            import output_parser
    finally:
        sys.path.remove(REF_PYTHON)
    s, _ = case_system("hexane_small")
    bl = _blocks()
    bv = output.block_values(s, bl)
    info = output_parser.parse(output.summary_text(s, bl))
    mols = info["Number of molecules"][s.molecule.name]
    got = mols["Average loading absolute [molecules/unit cell]"]
    assert abs(got[0] - np.mean(bv["molecules"])) < 1e-9 and got[1] == "+/-"
    assert "Average loading excess [mol/kg framework]" in mols
    assert abs(info["Enthalpy of adsorption"]["[K]"][0] - np.mean(bv["enthalpy_K"])) < 1e-4
    assert abs(info["Average Widom Rosenbluth factor"]["Widom"][0] - 0.002) < 1e-9
    assert info["Average Henry coefficient"]["Henry"][0] > 0
