"""The Coulomb grid on the GPU (charged CO2 in the charged framework).

- rgpu_grid_build_coulomb reproduces the reference's Coulomb grid file and
  the oracle's grid; its lookups reproduce InterpolateCoulombGrid.
- With VDW and Coulomb grids the FP64 engine follows the oracle with the same
  grids move for move (Ewald Fourier part unchanged).
- The mixed engine's running host VDW and host real-space charge energies
  equal the sums of grid lookups at the final molecules.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from raspa2_b200 import native, systems, units

from golden_cases import load, system_of

pytestmark = pytest.mark.gpu


def plane_major(buf, npts):
    host = buf.cpu().numpy().reshape(npts[0] + 1, npts[1] + 1, npts[2] + 1, 8)
    return np.ascontiguousarray(np.moveaxis(host, 3, 0))


@pytest.fixture(scope="module")
def built(cuda):
    c = load("grid_co2_coulomb")
    s = system_of(c)
    g = native.GpuSystem(s, maxmol=4)
    m = c["meta"]
    n = np.array(m["n"])
    buf = torch.zeros(int(np.prod(n + 1)) * 8, dtype=torch.float32, device="cuda")
    g.grid_build_coulomb(n, m["size"], m["shift"], buf.data_ptr())
    torch.cuda.synchronize()
    return c, s, g, buf, plane_major(buf, n)


def test_coulomb_grid_matches_reference_file(built):
    c, s, g, buf, planes = built
    flat = planes.reshape(8, -1)
    got = flat[:, np.array(c["sample_index"])].T
    np.testing.assert_allclose(got, np.array(c["sample_values"]), rtol=2e-7, atol=1e-6)
    for m in range(8):
        ours = float(np.sum(flat[m].astype(np.float64)))
        assert abs(ours - c["plane_sums"][m]) <= 1e-6 * c["plane_abs_sums"][m] + 1e-6


def test_coulomb_grid_matches_oracle(built):
    c, s, g, buf, planes = built
    m = c["meta"]
    ref = O.Oracle.from_system(s).grid_build_coulomb(m["n"], m["size"], m["shift"])
    np.testing.assert_allclose(planes, ref, rtol=2e-7, atol=1e-5)


def test_coulomb_lookup_matches_reference(built):
    c, s, g, buf, planes = built
    m = c["meta"]
    pts = np.array(c["interp_points"])
    raw = native.grid_interpolate(buf.data_ptr(), m["n"], m["size"], m["shift"], m["cell"], pts)
    got = np.concatenate([systems.PSEUDO_ATOMS[name][2] * raw for name in c["types"]])
    np.testing.assert_allclose(got, np.array(c["interp_ref"]), rtol=2e-5, atol=1e-3)


SPACING = 0.25


def _gridded(s, seed, stream_id, mols):
    g = native.GpuSystem(s, maxmol=64, seed=seed, stream_id=stream_id)
    g.set_adsorbates(mols)
    geom = g.use_energy_grids(SPACING)
    return g, geom


def test_fp64_engine_with_coulomb_grid_follows_oracle(cuda):
    c = load("co2_config1")
    s = system_of(c)
    mols = np.array(c["molecules"])
    n = 300
    g, (npts, size, shift, cell) = _gridded(s, 777, 3, mols)
    e = native.Engine([g], precision=native.RGPU_FP64, threads=256, cluster=2)
    e.run(n)
    e.sync()
    st = g.state()
    o = O.Oracle.from_system(s, maxmol=64)
    types = sorted(set(int(t) for t in s.molecule_types()))
    o.set_grids({t: plane_major(g._grids[t], npts) for t in types}, npts, size, shift, cell)
    cbuf, nc = g._grids["coulomb"]
    o.set_coulomb_grid(plane_major(cbuf, nc), nc, size, shift, cell)
    o.set_molecules(mols)
    ost = O.MCState()
    o.mc_run(O.mc_params(s, 777, 3), ost, 0, n)
    assert st["status"] == 0
    np.testing.assert_array_equal(st["counters"][0:4], np.array(ost.attempts[:4]))
    np.testing.assert_array_equal(st["counters"][4:8], np.array(ost.accepted[:4]))
    assert st["nmol"] == o.nmol
    np.testing.assert_allclose(g.adsorbates(), o.molecules(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(st["energy"][:6], np.array(ost.u), rtol=1e-9, atol=1e-6)


def test_mixed_engine_with_coulomb_grid_matches_lookups(cuda):
    c = load("co2_config1")
    s = system_of(c)
    g, (npts, size, shift, cell) = _gridded(s, 31, 5, np.zeros((0, 3, 3)))
    e = native.Engine([g], precision=native.RGPU_MIXED, threads=512, cluster=2)
    e.run(3000)
    e.sync()
    st = g.state()
    assert st["status"] == 0 and st["nmol"] > 3
    x = g.adsorbates()
    types = s.molecule_types()
    q = s.molecule.charges()
    cbuf, nc = g._grids["coulomb"]
    hv = sum(native.grid_interpolate(g._grids[int(types[a])].data_ptr(), npts, size, shift, cell, x[:, a]).sum()
             for a in range(x.shape[1]))
    hc = sum(q[a] * native.grid_interpolate(cbuf.data_ptr(), nc, size, shift, cell, x[:, a]).sum()
             for a in range(x.shape[1]))
    kT = units.K_B * s.temperature
    assert abs(st["energy"][0] - hv) <= 1e-9 * abs(hv) + 1e-6 * kT
    assert abs(st["energy"][2] - hc) <= 1e-9 * abs(hc) + 1e-6 * kT
