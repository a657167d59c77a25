"""The drop-in: the reference program itself, with its per-call energy
routines routed to the GPU, against the stock reference program.

oracle/_ref/simulate_gpu is the reference's own objects linked with
raspa2_b200/bridge/raspa_gpu_bridge.c under the linker's --wrap option
(oracle/Makefile, target `dropin`): the reference's MC loop (src/mc_moves.c,
src/cbmc.c) runs unchanged and every energy-at-a-position, move-difference
and Ewald Fourier call lands in libraspa_gpu. With one RandomSeed both
programs take the same decisions: the counter blocks of every move type are
equal, and the energies they print agree to 1e-9 relative (the GPU sums in
another order than the CPU, so the last digits differ).

co2_triclinic runs in a triclinic cell (angles 80, 95, 110 degrees). The
*_grid cases run with the GRID framework model (UseTabularGrid): the
stock program first makes the grids (SimulationType MakeGrid), then both
programs read them; the bridge reads the same files into device memory
with the library's grid-file reader. The hexane cases grow flexible chains
by the reference's CBMC with the external energies of every bead on the
GPU.

Both binaries are built where the reference's sources are (build()); the
test is skipped when they are absent.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from raspa2_b200 import raspa_io, systems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
SIMULATE = os.path.join(REF, "simulate")
SIMULATE_GPU = os.path.join(REF, "simulate_gpu")
RTOL = 1e-9

def hexane_small():
    return systems.hexane_system(seed=4, n_atoms=1200, cell=26.0)


# case: (system builder, cycles, grid spacing or None)
CASES = {
    "co2_tiny": (lambda: systems.tiny_co2_system(), 60, None),
    "co2_config1": (lambda: systems.co2_system(seed=1), 12, None),
    "methane_config0": (lambda: systems.methane_system(seed=0), 12, None),
    "hexane_small": (hexane_small, 12, None),
    "co2_triclinic": (lambda: systems.co2_triclinic_system(), 12, None),
    "co2_triclinic_grid": (lambda: systems.co2_triclinic_system(), 12, 1.0),
    "co2_config1_grid": (lambda: systems.co2_system(seed=1), 12, 0.5),
    "methane_config0_grid": (lambda: systems.methane_system(seed=0), 12, 0.5),
    "hexane_small_grid": (hexane_small, 12, 0.5),
}


def make_grids(s, d, spacing):
    """The reference's MakeGrid run of the stock program: grid files under
    d/share/raspa/grids (RASPA_DIR=d) for every pseudo-atom of the molecule."""
    types = sorted({systems.TYPE_ORDER[int(t)] for t in s.molecule_types()})
    grid = {"types": types, "spacing": spacing}
    raspa_io.write_inputs(s, d, simulation_type="MakeGrid", grid=grid)
    os.makedirs(os.path.join(d, "share", "raspa", "grids"), exist_ok=True)
    r = subprocess.run([SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True, timeout=1200,
                       env=dict(os.environ, RASPA_DIR=d))
    assert r.returncode == 0, r.stderr[-2000:]
    return dict(grid, use=True)


def run(binary, d, env=None):
    r = subprocess.run([binary, "-i", "simulation.input"], cwd=d, capture_output=True, text=True, timeout=1200,
                       env=env)
    assert r.returncode == 0, (binary, r.stderr[-2000:])
    out = os.path.join(d, "Output", "System_0")
    return open(os.path.join(out, os.listdir(out)[0])).read(), r.stderr


def summary(txt):
    cur = [float(x) for x in re.findall(r"Current total potential energy:\s+([-\d.eE+]+) \[K\]", txt)]
    tot = [float(x) for x in re.findall(r"^Total energy:\s+([-\d.eE+]+)", txt, re.M)]
    # the counter blocks of the moves (tries, successes, acceptances and the
    # adapted step sizes that follow from them)
    moves = re.findall(r"Performance of the (translation|rotation|swap addition|swap deletion|reinsertion) move:\n"
                       r"=+\n(.*?)\n\n", txt, re.S)
    return np.array(cur), np.array(tot), moves


@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_program_on_gpu_matches_stock_reference(cuda, case, tmp_path):
    if not (os.path.exists(SIMULATE) and os.path.exists(SIMULATE_GPU)):
        pytest.skip("reference programs not built (make -C oracle ref dropin)")
    build, cycles, spacing = CASES[case]
    s = build()
    kw = dict(cycles=cycles, init_cycles=0, print_every=max(1, cycles // 4), seed=4242)
    env = dict(os.environ)
    if spacing:
        d_grid = str(tmp_path / "grids")
        kw["grid"] = make_grids(s, d_grid, spacing)
        env["RASPA_DIR"] = d_grid
    d_cpu = raspa_io.write_inputs(s, str(tmp_path / "cpu"), **kw)
    d_gpu = raspa_io.write_inputs(s, str(tmp_path / "gpu"), **kw)
    txt_cpu, _ = run(SIMULATE, d_cpu, env=env)
    txt_gpu, err = run(SIMULATE_GPU, d_gpu, env=dict(env, RASPA_GPU_BRIDGE_STATS="1"))
    # the GPU did the work: the bridge reports its device calls
    m = re.search(r"point energies (\d+), move differences (\d+), Ewald (\d+)", err)
    assert m and int(m.group(1)) > 0 and int(m.group(2)) > 0, err[-500:]
    if s.ewald:
        assert int(m.group(3)) > 0
    cur_c, tot_c, mv_c = summary(txt_cpu)
    cur_g, tot_g, mv_g = summary(txt_gpu)
    assert len(mv_c) >= 3 and mv_c == mv_g, (mv_c, mv_g)
    assert re.search(r"accepted: [1-9]", dict(mv_c)["swap addition"])
    assert len(cur_c) == len(cur_g) > 0
    scale = np.abs(cur_c).max() + 1.0
    np.testing.assert_allclose(cur_g, cur_c, rtol=RTOL, atol=RTOL * scale)
    # running total and recomputed total at the end: the same on both
    assert len(tot_c) == len(tot_g) >= 2
    np.testing.assert_allclose(tot_g, tot_c, rtol=RTOL, atol=RTOL * scale)
    # and the GPU run's running energy agrees with the reference's own
    # recomputation from scratch (its energy-drift check)
    np.testing.assert_allclose(tot_g[-2], tot_g[-1], rtol=RTOL, atol=RTOL * scale)


@pytest.mark.parametrize("case,spacing", [("methane_config0", 0.5), ("co2_config1", 1.0), ("co2_triclinic", 1.0)])
def test_make_grid_on_gpu_writes_the_reference_grid_files(cuda, case, spacing, tmp_path):
    """SimulationType MakeGrid: simulate_gpu builds the grids on the GPU and
    writes the same files as the stock program (same paths, headers equal
    byte for byte, values equal to FP32 rounding of differently ordered
    framework sums)."""
    if not (os.path.exists(SIMULATE) and os.path.exists(SIMULATE_GPU)):
        pytest.skip("reference programs not built (make -C oracle ref dropin)")
    build, _, _ = CASES[case]
    s = build()
    types = sorted({systems.TYPE_ORDER[int(t)] for t in s.molecule_types()})
    out = {}
    for name, binary in (("cpu", SIMULATE), ("gpu", SIMULATE_GPU)):
        d = str(tmp_path / name)
        raspa_io.write_inputs(s, d, simulation_type="MakeGrid", grid={"types": types, "spacing": spacing})
        os.makedirs(os.path.join(d, "share", "raspa", "grids"), exist_ok=True)
        r = subprocess.run([binary, "-i", "simulation.input"], cwd=d, capture_output=True, text=True, timeout=1200,
                           env=dict(os.environ, RASPA_DIR=d))
        assert r.returncode == 0, (binary, r.stderr[-2000:])
        root = os.path.join(d, "share", "raspa", "grids")
        out[name] = {os.path.relpath(os.path.join(p, f), root): os.path.join(p, f)
                     for p, _, fs in os.walk(root) for f in fs if f.endswith(".grid")}
    assert sorted(out["cpu"]) == sorted(out["gpu"]) and len(out["cpu"]) == len(types) + (1 if s.ewald else 0)
    for rel, fc in out["cpu"].items():
        coulomb = "Electrostatics" in rel
        hb = 136 if coulomb else 128
        with open(fc, "rb") as a, open(out["gpu"][rel], "rb") as b:
            ba, bb = a.read(), b.read()
        assert len(ba) == len(bb) and ba[:hb] == bb[:hb], rel
        va = np.frombuffer(ba, np.float32, offset=hb).astype(np.float64)
        vb = np.frombuffer(bb, np.float32, offset=hb).astype(np.float64)
        err = np.abs(va - vb) / (np.abs(va) + 1.0)
        assert err.max() <= 1e-5, (rel, float(err.max()), int(err.argmax()))
