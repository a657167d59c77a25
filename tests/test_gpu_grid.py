"""GPU energy-grid construction and tricubic lookup against the reference's
grid file and InterpolateVDWGrid values (tests/golden/grid_methane.json)."""
import numpy as np
import pytest

from oracle import oracle as O
from raspa2_b200 import native, systems

from golden_cases import load, system_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grid(cuda):
    import torch
    c = load("grid_methane")
    s = system_of(c)
    g = native.GpuSystem(s, maxmol=4)
    m = c["meta"]
    n = np.array(m["n"])
    buf = torch.zeros(int(np.prod(n + 1)) * 8, dtype=torch.float32, device="cuda")
    t = systems.TYPE_ORDER.index("CH4_sp3")
    g.grid_build(t, n, m["size"], m["shift"], buf.data_ptr())
    torch.cuda.synchronize()
    host = buf.cpu().numpy().reshape(n[0] + 1, n[1] + 1, n[2] + 1, 8)
    return c, s, g, buf, host


def test_grid_matches_reference_file(grid):
    c, s, g, buf, host = grid
    planes = np.moveaxis(host, 3, 0).reshape(8, -1)      # device point-major -> file plane-major
    got = planes[:, np.array(c["sample_index"])].T
    np.testing.assert_allclose(got, np.array(c["sample_values"]), rtol=2e-7, atol=1e-6)
    sums = [float(np.sum(planes[k].astype(np.float64))) for k in range(8)]
    np.testing.assert_allclose(sums, c["plane_sums"], rtol=1e-6)


def test_grid_matches_oracle(grid):
    c, s, g, buf, host = grid
    m = c["meta"]
    o = O.Oracle.from_system(s)
    t = systems.TYPE_ORDER.index("CH4_sp3")
    ref = o.grid_build(t, m["n"], m["size"], m["shift"])
    np.testing.assert_allclose(np.moveaxis(host, 3, 0), ref, rtol=2e-7, atol=1e-5)


def test_interpolation_matches_oracle_on_same_grid(grid):
    """GPU lookup = oracle lookup on the identical (GPU-built) grid."""
    c, s, g, buf, host = grid
    m = c["meta"]
    pts = np.array(c["interp_points"])
    got = native.grid_interpolate(buf.data_ptr(), m["n"], m["size"], m["shift"], m["cell"], pts)
    planes = np.ascontiguousarray(np.moveaxis(host, 3, 0))
    ref = [O.grid_interpolate(planes, m["n"], m["size"], m["shift"], m["cell"], p) for p in pts]
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-9)


def test_interpolation_matches_reference(grid):
    """Against InterpolateVDWGrid on the reference's own grid file. The two
    grids agree to FP32 rounding (framework summation order differs), and the
    Hermite sum of a cell near the repulsive wall cancels by up to ~100x, so
    the bound is 2e-5 relative (1e-6 absolute floor)."""
    c, s, g, buf, host = grid
    m = c["meta"]
    pts = np.array(c["interp_points"])
    got = native.grid_interpolate(buf.data_ptr(), m["n"], m["size"], m["shift"], m["cell"], pts)
    np.testing.assert_allclose(got, c["interp_ref"], rtol=2e-5, atol=1e-6)
