"""rgpu_grid_interpolate_noalloc: the grid lookup through the library's static
device scratch gives the same values as rgpu_grid_interpolate (which allocates
its buffers per call), on two calls in a row, and refuses more points than
the scratch holds. Self-contained so that it passes alone in a fresh process
as well as after the rest of the suite."""
import numpy as np
import pytest

from raspa2_b200 import native, systems

from golden_cases import load, system_of

pytestmark = pytest.mark.gpu

RTOL = 1e-12   # same kernel on the same grid; only the buffers differ


@pytest.fixture(scope="module")
def grid(cuda):
    import torch
    c = load("grid_methane")
    s = system_of(c)
    g = native.GpuSystem(s, maxmol=4)
    m = c["meta"]
    n = np.array(m["n"])
    buf = torch.zeros(int(np.prod(n + 1)) * 8, dtype=torch.float32, device="cuda")
    g.grid_build(systems.TYPE_ORDER.index("CH4_sp3"), n, m["size"], m["shift"], buf.data_ptr())
    torch.cuda.synchronize()
    return m, g, buf


def _points(m, n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 1.0, (n, 3)) * np.array(m["cell"]) * np.array(m["ncell"])


def test_noalloc_matches_allocating_lookup_twice(grid):
    m, g, buf = grid
    args = (buf.data_ptr(), m["n"], m["size"], m["shift"], m["cell"])
    # the second call has fewer points than the first: stale results of the
    # first call must not leak into it
    for n, seed in ((3000, 11), (1234, 12)):
        pts = _points(m, n, seed)
        got = native.grid_interpolate_noalloc(*args, pts)
        ref = native.grid_interpolate(*args, pts)
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=0.0)


def test_noalloc_full_capacity(grid):
    m, g, buf = grid
    args = (buf.data_ptr(), m["n"], m["size"], m["shift"], m["cell"])
    pts = _points(m, native.RGPU_NOALLOC_MAX_POINTS, 13)
    np.testing.assert_allclose(native.grid_interpolate_noalloc(*args, pts), native.grid_interpolate(*args, pts),
                               rtol=RTOL, atol=0.0)


def test_noalloc_rejects_more_points_than_scratch(grid):
    m, g, buf = grid
    pts = _points(m, native.RGPU_NOALLOC_MAX_POINTS + 1, 14)
    with pytest.raises(native.NativeError, match="RGPU_NOALLOC_MAX_POINTS"):
        native.grid_interpolate_noalloc(buf.data_ptr(), m["n"], m["size"], m["shift"], m["cell"], pts)


def test_noalloc_allocates_no_device_memory(grid):
    """The property the entry point exists for: after the first call (which
    may load the module's code), further calls leave the device's free
    memory unchanged."""
    import torch
    m, g, buf = grid
    args = (buf.data_ptr(), m["n"], m["size"], m["shift"], m["cell"])
    pts = _points(m, native.RGPU_NOALLOC_MAX_POINTS, 15)
    first = native.grid_interpolate_noalloc(*args, pts)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        np.testing.assert_array_equal(native.grid_interpolate_noalloc(*args, pts), first)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
