"""The oracle's flexible-chain CBMC (CPU): bookkeeping of the
intramolecular energy, fixed bond lengths, and the sampled bend-angle and
torsion distributions of the grown chains."""
import numpy as np

from oracle import oracle as O
from raspa2_b200 import systems, units


def test_chain_growth_and_bookkeeping():
    s = systems.hexane_system(seed=4, n_atoms=1200, cell=26.0, pressure=1e6)
    o = O.Oracle.from_system(s, maxmol=64)
    o.set_molecules(np.zeros((0, 6, 3)))
    st = O.MCState()
    o.mc_run(O.mc_params(s, 777, 3), st, 0, 3000)
    assert o.nmol > 5
    # running energies equal a recomputation
    np.testing.assert_allclose(st.u_intra, o.intra_energy(), rtol=1e-9)
    np.testing.assert_allclose(np.array(st.u)[:2], o.total_energy()[:2], rtol=1e-9)
    x = o.molecules()
    np.testing.assert_allclose(np.linalg.norm(np.diff(x, axis=1), axis=2), 1.54, atol=1e-9)
    # bend angles spread about 114 degrees with the harmonic width
    u = x[:, :-2] - x[:, 1:-1]
    v = x[:, 2:] - x[:, 1:-1]
    th = np.degrees(np.arccos(np.sum(u * v, -1) / np.linalg.norm(u, axis=-1) / np.linalg.norm(v, axis=-1)))
    sigma = np.degrees(1.0 / np.sqrt(units.beta(s.temperature) * 62500.0 * units.K_B))
    assert abs(th.mean() - 114.0) < 3.0 * sigma
    assert 0.5 * sigma < th.std() < 2.0 * sigma


def test_chain_growth_on_energy_grids():
    """With energy grids the oracle's running host VDW energy is the sum of
    grid lookups at the beads (a coarse 0.5 A grid keeps this fast; how
    closely lookups follow the pair sums at production spacing is checked on
    the GPU, where the grids are cheap to build)."""
    s = systems.hexane_system(seed=4, n_atoms=1200, cell=26.0, pressure=1e6)
    o = O.Oracle.from_system(s, maxmol=64)
    uc = np.asarray(s.unit_cell, float)
    npts = (uc / 0.5).astype(np.int32)
    types = sorted(set(int(t) for t in s.molecule_types()))
    grids = {t: o.grid_build(t, npts, uc, np.zeros(3)) for t in types}
    o.set_grids(grids, npts, uc, np.zeros(3), uc)
    o.set_molecules(np.zeros((0, 6, 3)))
    st = O.MCState()
    o.mc_run(O.mc_params(s, 91, 2), st, 0, 600)
    assert o.nmol > 3
    with_grids = o.total_energy()[0]
    np.testing.assert_allclose(st.u[0], with_grids, rtol=1e-9)
    x = o.molecules()
    look = sum(O.grid_interpolate(grids[int(s.molecule_types()[a])], npts, uc, np.zeros(3), uc, p)
               for a in range(6) for p in x[:, a])
    np.testing.assert_allclose(look, with_grids, rtol=1e-12)
    o.set_grids(None, None, None, None, None)
    assert o.total_energy()[0] != with_grids     # the pair sums are back
