"""Flexible chains (united-atom n-hexane): the FP64 engine follows the
oracle's GCMC trajectory move for move (CBMC growth bead by bead with
sampled bends and torsions, translation, rotation, reinsertion, swaps), with
the reference's bonded-trial scheme (chain_scheme 0) and with independent
draws (chain_scheme 1), for CTA sizes of 64 and 256 threads and clusters of
1 to 8 CTAs; and the mixed engine's running energies, the intramolecular
part included, agree with a full recomputation."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from raspa2_b200 import native, systems, units

pytestmark = pytest.mark.gpu


def small_hexane(pressure=1e6):
    return systems.hexane_system(seed=4, n_atoms=1200, cell=26.0, pressure=pressure)


@pytest.mark.parametrize("threads,cluster,scheme", [(256, 1, 0), (256, 2, 0), (64, 1, 0), (64, 3, 0), (256, 8, 0),
                                                     (256, 2, 1), (64, 3, 1)])
def test_fp64_engine_follows_oracle_with_chains(cuda, threads, cluster, scheme):
    s = small_hexane()
    # independent draws carry no torsion factor: their ideal-gas weight is ~1.1
    s = dataclasses.replace(s, chain_scheme=scheme, ideal_gas_rosenbluth=s.ideal_gas_rosenbluth if scheme == 0 else 1.1)
    n = 1500
    g = native.GpuSystem(s, maxmol=64, seed=777, stream_id=3)
    g.set_adsorbates(np.zeros((0, 6, 3)))
    e = native.Engine([g], precision=native.RGPU_FP64, threads=threads, cluster=cluster)
    e.run(n)
    e.sync()
    st = g.state()
    o = O.Oracle.from_system(s, maxmol=64)
    o.set_molecules(np.zeros((0, 6, 3)))
    ost = O.MCState()
    o.mc_run(O.mc_params(s, 777, 3), ost, 0, n)
    assert st["status"] == 0
    np.testing.assert_array_equal(st["counters"][0:4], np.array(ost.attempts[:4]))
    np.testing.assert_array_equal(st["counters"][4:8], np.array(ost.accepted[:4]))
    assert st["counters"][18] == ost.attempts[4] and st["counters"][19] == ost.accepted[4]
    assert st["nmol"] == o.nmol > 5
    np.testing.assert_allclose(g.adsorbates(), o.molecules(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(st["energy"][[0, 1]], np.array(ost.u)[:2], rtol=1e-9, atol=1e-6)
    np.testing.assert_allclose(st["energy"][6], ost.u_intra, rtol=1e-9, atol=1e-6)


def test_mixed_engine_chain_energies_track_recomputation(cuda):
    s = small_hexane()
    g = native.GpuSystem(s, maxmol=64, seed=11, stream_id=1)
    g.set_adsorbates(np.zeros((0, 6, 3)))
    e = native.Engine([g], precision=native.RGPU_MIXED, threads=256, cluster=2)
    e.run(3000)
    e.sync()
    st = g.state()
    assert st["nmol"] > 5 and st["status"] == 0
    tot = g.total_energy()
    kT = units.K_B * s.temperature
    assert abs(st["energy"][0] - tot[0]) <= 1e-6 * abs(tot[0]) + 1e-3 * kT
    assert abs(st["energy"][1] - tot[1]) <= 1e-6 * abs(tot[1]) + 1e-3 * kT
    assert abs(st["energy"][6] - g.intra_energy()) <= 1e-9 * abs(g.intra_energy()) + 1e-6 * kT
    # the chains keep their bond lengths
    x = g.adsorbates()
    np.testing.assert_allclose(np.linalg.norm(np.diff(x, axis=1), axis=2), 1.54, atol=1e-9)
