"""Energy grids on the engine's path (grid-accelerated CBMC of united-atom
n-hexane, UseTabularGrid in the reference): the host VDW energy of a bead is
the tricubic lookup in its pseudo-atom type's grid instead of the pair sum
over the framework.

- The FP64 engine with grids follows the oracle with the same grids move for
  move (the grids are built on the GPU and handed to both).
- The mixed engine's running host VDW energy equals the sum of grid lookups
  at the final beads (it is a sum of lookups, so only FP64 rounding of the
  running sum separates them).
- Those lookups agree with the direct FP64 pair sums per bead within the
  interpolation error of a 0.15 A grid.
"""
import numpy as np
import pytest

from oracle import oracle as O
from raspa2_b200 import native, systems, units

pytestmark = pytest.mark.gpu

SPACING = 0.15


def small_hexane(pressure=1e6):
    return systems.hexane_system(seed=4, n_atoms=1200, cell=26.0, pressure=pressure)


def plane_major(g, npts, t):
    host = g._grids[t].cpu().numpy().reshape(npts[0] + 1, npts[1] + 1, npts[2] + 1, 8)
    return np.ascontiguousarray(np.moveaxis(host, 3, 0))


@pytest.mark.parametrize("cluster", [1, 2])
def test_fp64_engine_with_grids_follows_oracle(cuda, cluster):
    s = small_hexane()
    n = 1500
    g = native.GpuSystem(s, maxmol=64, seed=778, stream_id=5)
    g.set_adsorbates(np.zeros((0, 6, 3)))
    npts, size, shift, cell = g.use_energy_grids(SPACING)
    e = native.Engine([g], precision=native.RGPU_FP64, threads=256, cluster=cluster)
    e.run(n)
    e.sync()
    st = g.state()
    o = O.Oracle.from_system(s, maxmol=64)
    o.set_grids({t: plane_major(g, npts, t) for t in g._grids}, npts, size, shift, cell)
    o.set_molecules(np.zeros((0, 6, 3)))
    ost = O.MCState()
    o.mc_run(O.mc_params(s, 778, 5), ost, 0, n)
    assert st["status"] == 0
    np.testing.assert_array_equal(st["counters"][0:4], np.array(ost.attempts[:4]))
    np.testing.assert_array_equal(st["counters"][4:8], np.array(ost.accepted[:4]))
    assert st["counters"][18] == ost.attempts[4] and st["counters"][19] == ost.accepted[4]
    assert st["nmol"] == o.nmol > 5
    np.testing.assert_allclose(g.adsorbates(), o.molecules(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(st["energy"][[0, 1]], np.array(ost.u)[:2], rtol=1e-9, atol=1e-6)
    np.testing.assert_allclose(st["energy"][6], ost.u_intra, rtol=1e-9, atol=1e-6)


def test_mixed_engine_with_grids_matches_lookups_and_direct_sums(cuda):
    s = small_hexane()
    g = native.GpuSystem(s, maxmol=64, seed=12, stream_id=1)
    g.set_adsorbates(np.zeros((0, 6, 3)))
    npts, size, shift, cell = g.use_energy_grids(SPACING)
    e = native.Engine([g], precision=native.RGPU_MIXED, threads=256, cluster=2)
    e.run(3000)
    e.sync()
    st = g.state()
    assert st["nmol"] > 5 and st["status"] == 0
    kT = units.K_B * s.temperature
    x = g.adsorbates()
    types = s.molecule_types()
    look = np.stack([native.grid_interpolate(g._grids[int(types[a])].data_ptr(), npts, size, shift, cell, x[:, a])
                     for a in range(x.shape[1])], axis=1)
    assert abs(st["energy"][0] - look.sum()) <= 1e-9 * np.abs(look).sum() + 1e-6 * kT
    # direct FP64 pair sums per bead (the engine's own energy routine, no grids)
    direct = np.stack([g.bead_energies(x[:, a], a, -1)[:, 0] for a in range(x.shape[1])], axis=1)
    err = np.abs(look - direct)
    # tricubic Hermite error at 0.15 A: well under 1 % of the bead energy plus
    # 0.01 k_B T
    assert np.all(err <= 1e-2 * np.abs(direct) + 1e-2 * kT), (err.max() / kT, np.abs(direct).max() / kT)
    assert abs(look.sum() - direct.sum()) <= 1e-3 * np.abs(direct).sum() + 0.1 * kT
    # the direct total of the engine's configuration, switched back to pair sums
    g.set_grids(None, None, None, None, None)
    assert abs(g.total_energy()[0] - direct.sum()) <= 1e-9 * np.abs(direct).sum() + 1e-6 * kT


def test_grid_loading_matches_direct_sums(cuda):
    """GCMC of n-hexane at 3e4 Pa: the average loading with 0.1 A grids equals
    the loading with direct pair sums within the combined statistical error
    (64 independent replicas each)."""
    import dataclasses
    from test_gpu_stats import engine_ideal_gas_rosenbluth
    s = small_hexane(pressure=3e4)
    w, _ = engine_ideal_gas_rosenbluth(s.molecule, s.temperature)
    s = dataclasses.replace(s, ideal_gas_rosenbluth=w)
    equil, prod, nrep = 50000, 100000, 64
    loads = {}
    for grids in (False, True):
        gs = []
        for i in range(nrep):
            g = native.GpuSystem(s, maxmol=32, seed=(9000 if grids else 7000) + i, stream_id=i)
            g.set_adsorbates(np.zeros((0, 6, 3)))
            if grids:
                if gs:
                    g.use_energy_grids(0.1, like=gs[0])
                else:
                    g.use_energy_grids(0.1)
            g.set_limits(equil + prod, equil)
            gs.append(g)
        e = native.Engine(gs, precision=native.RGPU_MIXED)
        e.run(equil + prod)
        e.sync()
        loads[grids] = np.array([g.averages()["loading"] for g in gs])
    a, b = loads[False], loads[True]
    se = np.hypot(a.std(ddof=1), b.std(ddof=1)) / np.sqrt(nrep)
    assert abs(a.mean() - b.mean()) <= 4.0 * se, (a.mean(), b.mean(), se)
