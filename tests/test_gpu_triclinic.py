"""A triclinic box (cell angles 80, 95, 110 degrees; the CO2 model of
config 1): the reference's triclinic minimum image, wave vectors and random
positions on the GPU.

- The per-call entry points against the reference's own outputs for this
  box are in tests/test_gpu_parity.py (case co2_triclinic).
- The FP64 engine follows the oracle's GCMC trajectory move for move (the
  oracle is pinned to the reference for this box by
  tests/test_oracle_golden.py).
- The mixed engine's running energies equal an FP64 recomputation.
- Energy grids of the triclinic cell built on the GPU equal the
  reference's, and their lookups the reference's TRICLINIC branch.
"""
import numpy as np
import pytest

from raspa2_b200 import native, systems, units

from golden_cases import load, system_of
from test_gpu_engine import engine_run, oracle_run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cluster", [1, 2, 3])
def test_fp64_engine_reproduces_oracle_trajectory(cuda, cluster):
    c = load("co2_triclinic")
    s = system_of(c)
    assert s.triclinic
    mols = np.array(c["molecules"])
    n = 300
    g, st = engine_run(s, mols, n, native.RGPU_FP64, cluster=cluster)
    o, ost = oracle_run(s, mols, n)
    assert st["status"] == 0 and st["step"] == n
    np.testing.assert_array_equal(st["counters"][0:4], np.array(ost.attempts[:4]))
    np.testing.assert_array_equal(st["counters"][4:8], np.array(ost.accepted[:4]))
    assert st["counters"][4:8].sum() > 20
    assert st["nmol"] == o.nmol
    np.testing.assert_allclose(g.adsorbates(), o.molecules(), rtol=0, atol=1e-10)
    np.testing.assert_allclose(st["energy"][:6], np.array(ost.u), rtol=1e-9, atol=1e-6)


@pytest.mark.parametrize("precision,tol", [(native.RGPU_FP64, 1e-10), (native.RGPU_MIXED, 1e-6)])
def test_running_energy_equals_recomputation(cuda, precision, tol):
    c = load("co2_triclinic")
    s = system_of(c)
    g = native.GpuSystem(s, maxmol=128, seed=5, stream_id=2)
    g.set_adsorbates(np.array(c["molecules"])[:4])
    e0 = g.total_energy()
    g.set_energy(np.concatenate([e0, [0, 0]]))
    eng = native.Engine([g], precision=precision, cluster=2)
    eng.run(2000)
    eng.sync()
    st = g.state()
    assert st["status"] == 0
    acc = st["counters"][4:8].sum()
    assert acc > 20 and st["nmol"] > 4
    e1 = g.total_energy()
    kT = units.K_B * s.temperature
    drift = np.abs(st["energy"][:6] - e1)
    scale = np.maximum(np.abs(e1), kT)
    assert np.all(drift <= tol * scale * max(1.0, acc / 100.0)), (st["energy"][:6], e1, drift / scale)


def test_grids_match_reference(cuda):
    """Grids of the triclinic cell built on the GPU over its enclosing box
    equal the reference's files (samples, plane sums), and with the GRID
    framework model the per-call energies are the reference's lookups, each
    point wrapped into the triclinic unit cell (tests/golden/grid_co2_triclinic.json)."""
    import torch
    c = load("grid_co2_triclinic")
    s = system_of(c)
    g = native.GpuSystem(s, maxmol=8)
    bufs = {}
    for kind, m in c["meta"].items():
        n = np.array(m["n"])
        buf = torch.zeros(int(np.prod(n + 1)) * 8, dtype=torch.float32, device="cuda")
        if kind == "coulomb":
            g.grid_build_coulomb(n, m["size"], m["shift"], buf.data_ptr())
        else:
            g.grid_build(systems.TYPE_ORDER.index(kind), n, m["size"], m["shift"], buf.data_ptr())
        torch.cuda.synchronize()
        host = buf.cpu().numpy().reshape(n[0] + 1, n[1] + 1, n[2] + 1, 8)
        flat = np.moveaxis(host, 3, 0).reshape(8, -1)
        smp = c["samples"][kind]
        np.testing.assert_allclose(flat[:, np.array(smp["index"])].T, np.array(smp["values"]), rtol=2e-7, atol=1e-6)
        for q in range(8):
            ours = float(np.sum(flat[q].astype(np.float64)))
            assert abs(ours - c["plane_sums"][kind]["sum"][q]) <= 1e-6 * c["plane_sums"][kind]["abs"][q] + 1e-6
        bufs[kind] = buf
    mc = c["meta"]["coulomb"]
    g.set_coulomb_grid(bufs["coulomb"].data_ptr(), mc["n"], mc["size"], mc["shift"], mc["cell"])
    names = [systems.TYPE_ORDER[int(t)] for t in s.molecule_types()]
    m0 = c["meta"][names[0]]
    g.set_grids([bufs[nm].data_ptr() for nm in names], m0["n"], m0["size"], m0["shift"], m0["cell"])
    g.set_framework_model(native.RGPU_FRAMEWORK_GRID)
    pts = np.array(c["points"])
    for a, nm in enumerate(names):
        got = g.bead_energies(pts, a, -1)
        np.testing.assert_allclose(got[:, 0], c["interp_ref"][nm]["vdw"], rtol=2e-5, atol=1e-3)
        np.testing.assert_allclose(got[:, 1], c["interp_ref"][nm]["coulomb"], rtol=2e-5, atol=1e-3)


def test_fp64_engine_with_grids_follows_oracle(cuda):
    """VDW and Coulomb grids of the triclinic cell (built on the GPU at
    0.25 A, given to the oracle plane-major): the FP64 engine with grids
    follows the oracle with the same grids move for move. (At 0.5 A the
    interpolated Coulomb grid has deep artificial wells next to framework
    charges, whose Boltzmann factors overflow.)"""
    from oracle import oracle as O
    c = load("co2_triclinic")
    s = system_of(c)
    mols = np.array(c["molecules"])
    g = native.GpuSystem(s, maxmol=64, seed=777, stream_id=3)
    g.set_adsorbates(mols)
    npts, size, shift, cell = g.use_energy_grids(0.25)
    e = native.Engine([g], precision=native.RGPU_FP64, threads=256, cluster=2)
    e.run(300)
    e.sync()
    st = g.state()

    def planes(buf, n):
        host = buf.cpu().numpy().reshape(n[0] + 1, n[1] + 1, n[2] + 1, 8)
        return np.ascontiguousarray(np.moveaxis(host, 3, 0))

    o = O.Oracle.from_system(s, maxmol=64)
    types = sorted(set(int(t) for t in s.molecule_types()))
    o.set_grids({t: planes(g._grids[t], npts) for t in types}, npts, size, shift, cell)
    cbuf, nc = g._grids["coulomb"]
    o.set_coulomb_grid(planes(cbuf, nc), nc, size, shift, cell)
    o.set_molecules(mols)
    ost = O.MCState()
    o.mc_run(O.mc_params(s, 777, 3), ost, 0, 300)
    assert st["status"] == 0
    np.testing.assert_array_equal(st["counters"][0:4], np.array(ost.attempts[:4]))
    np.testing.assert_array_equal(st["counters"][4:8], np.array(ost.accepted[:4]))
    assert st["nmol"] == o.nmol
    np.testing.assert_allclose(g.adsorbates(), o.molecules(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(st["energy"][:6], np.array(ost.u), rtol=1e-9, atol=1e-6)
