"""Grid files on the GPU, and the GRID framework model of the per-call
energies.

- rgpu_grid_read_file puts the reference's own grid files
  (tests/golden/grid_files/, written by MakeGrid) on the device in the device
  layout bit for bit, and rgpu_grid_write_file writes them back byte for
  byte (ReadVDWGrid / WriteVDWGrid, src/grids.c:692-813; the Coulomb pair
  :815-977).
- With those grids and the GRID framework model, rgpu_bead_energies returns
  the reference's InterpolateVDWGrid and InterpolateCoulombGrid on the same
  files (src/framework_energy.c:73-77, :195-198).
- With adsorbates, the GRID model's bead energies, move differences and
  totals equal the oracle's grid branch on the same grids, and the FULL
  model returns to the pair sums.
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from raspa2_b200 import native, systems

from golden_cases import HERE, load, system_of

pytestmark = pytest.mark.gpu

FILES = os.path.join(HERE, "grid_files")


def file_planes(path, coulomb):
    h = native.grid_file_header(path, coulomb)
    n = np.array(h.npts) + 1
    return np.fromfile(path, dtype=np.float32, offset=136 if coulomb else 128).reshape(8, *n)


def plane_major(buf, npts):
    host = buf.cpu().numpy().reshape(npts[0] + 1, npts[1] + 1, npts[2] + 1, 8)
    return np.ascontiguousarray(np.moveaxis(host, 3, 0))


@pytest.fixture(scope="module")
def files(cuda):
    c = load("grid_co2_files")
    out = {}
    for kind, name in c["files"].items():
        path = os.path.join(FILES, name)
        coulomb = kind == "coulomb"
        n = np.array(native.grid_file_header(path, coulomb).npts)
        buf = torch.full((int(np.prod(n + 1)) * 8,), float("nan"), dtype=torch.float32, device="cuda")
        h = native.grid_read_file(path, buf.data_ptr(), buf.numel(), coulomb)
        out[kind] = (path, coulomb, h, buf)
    return c, out


def test_read_file_is_the_file_in_device_layout(files):
    c, out = files
    for kind, (path, coulomb, h, buf) in out.items():
        np.testing.assert_array_equal(plane_major(buf, list(h.npts)), file_planes(path, coulomb), err_msg=kind)


def test_write_file_round_trips_byte_for_byte(files, tmp_path):
    c, out = files
    for kind, (path, coulomb, h, buf) in out.items():
        dst = tmp_path / "share" / "raspa" / "grids" / os.path.basename(path)   # parents are created
        native.grid_write_file(str(dst), h, buf.data_ptr(), coulomb)
        with open(path, "rb") as a, open(dst, "rb") as b:
            assert a.read() == b.read(), kind


def test_read_file_refuses_a_small_buffer(files):
    c, out = files
    path, coulomb, h, buf = out["C_co2"]
    with pytest.raises(native.NativeError, match="error -1"):
        native.grid_read_file(path, buf.data_ptr(), buf.numel() - 1, coulomb)


def _grid_model(s, out):
    g = native.GpuSystem(s, maxmol=16)
    names = [systems.TYPE_ORDER[int(t)] for t in s.molecule_types()]
    _, _, hc, cbuf = out["coulomb"]
    g.set_coulomb_grid(cbuf.data_ptr(), list(hc.npts), list(hc.size), list(hc.shift), list(hc.unit_cell))
    h = out[names[0]][2]
    g.set_grids([out[nm][3].data_ptr() for nm in names], list(h.npts), list(h.size), list(h.shift),
                list(h.unit_cell))
    return g, names


@pytest.mark.parametrize("precision", [native.RGPU_FP64, native.RGPU_MIXED])
def test_grid_model_bead_energies_are_the_reference_lookups(files, precision):
    """The reference's lookups on its own files (values in the reference's
    internal energy unit). The two interpolants are the same cubic in another
    arrangement: they agree to FP64 rounding of terms up to ~1e8."""
    c, out = files
    s = system_of(c)
    g, names = _grid_model(s, out)
    pts = np.array(c["points"])
    full = g.bead_energies(pts, 0, -1, precision)
    g.set_framework_model(native.RGPU_FRAMEWORK_GRID)
    for a, nm in enumerate(names):
        got = g.bead_energies(pts, a, -1, precision)
        ref = c["interp_ref"][nm]
        np.testing.assert_allclose(got[:, 0], ref["vdw"], rtol=1e-9, atol=1e-5)
        np.testing.assert_allclose(got[:, 1], ref["coulomb"], rtol=1e-9, atol=1e-5)
        assert not got[:, 2:].any()
    # FULL again: the pair sums, which a 2 A grid does not reproduce
    g.set_framework_model(native.RGPU_FRAMEWORK_FULL)
    np.testing.assert_array_equal(g.bead_energies(pts, 0, -1, precision), full)


def test_grid_model_needs_grids(cuda):
    s = system_of(load("co2_config1"))
    g = native.GpuSystem(s, maxmol=4)
    with pytest.raises(native.NativeError, match="error -1"):
        g.set_framework_model(native.RGPU_FRAMEWORK_GRID)
    with pytest.raises(native.NativeError, match="error -1"):
        g.set_framework_model(7)


def test_grid_model_follows_the_oracle_grid_branch(cuda):
    """Bead energies, move differences and totals with adsorbates, on grids
    built on the GPU at 0.25 A and given to the oracle plane-major."""
    c = load("co2_config1")
    s = system_of(c)
    mols = np.array(c["molecules"])
    g = native.GpuSystem(s, maxmol=64)
    g.set_adsorbates(mols)
    npts, size, shift, cell = g.use_energy_grids(0.25)
    o = O.Oracle.from_system(s, maxmol=64)
    types = [int(t) for t in s.molecule_types()]
    o.set_grids({t: plane_major(g._grids[t], npts) for t in set(types)}, npts, size, shift, cell)
    cbuf, nc = g._grids["coulomb"]
    o.set_coulomb_grid(plane_major(cbuf, nc), nc, size, shift, cell)
    o.set_molecules(mols)
    g.set_framework_model(native.RGPU_FRAMEWORK_GRID)
    q = s.molecule.charges()
    for pt in c["points"]:
        got = g.bead_energies([pt["p"]], pt["atom"], pt["exclude"])[0]
        ref = o.point(types[pt["atom"]], float(q[pt["atom"]]), np.array(pt["p"]), pt["exclude"])
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-6)
        mixed = g.bead_energies([pt["p"]], pt["atom"], pt["exclude"], native.RGPU_MIXED)[0]
        np.testing.assert_allclose(mixed[:2], ref[:2], rtol=1e-12, atol=1e-9)   # the lookups are FP64
    compared = 0
    for mv in c["moves"]:
        new = np.array(mv["new"])
        ov, dl = g.move_difference(mv["m"], new)
        ov2, dl2 = o.move_delta(mv["m"], new)
        if ov2:
            continue
        compared += 1
        assert not ov
        np.testing.assert_allclose([dl[0], dl[2], dl[1], dl[3]], dl2, rtol=1e-9, atol=1e-6)
    assert compared >= 3
    np.testing.assert_allclose(g.total_energy(), o.total_energy(), rtol=1e-9, atol=1e-6)
