"""RGPU_MIXED_CC64: the mixed engine with every pair's distance, cut-off test
and real-space charge-charge term (erfc(alpha r)/r, src/potentials.c:12471)
in FP64, and the Fourier phases exp(ik.r) and dS(k) (src/ewald.c:7155-7306)
in FP64; LJ terms stay FP32.

- Same random stream: it takes the FP64 engine's decisions.
- Its running energies drift from an FP64 recomputation by less than the
  mixed engine's on the same runs. The charge terms carry most of the mixed
  engine's error: the real-space sums cancel by up to ~100x over the +-1.2 e
  framework charges, and the host Fourier term multiplies each dS(k) by the
  framework's S(k).
- It covers rigid molecules without energy grids; anything else is refused.
"""
import numpy as np
import pytest

from raspa2_b200 import native, systems, units

from golden_cases import load, system_of
from test_gpu_engine import engine_run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,n", [("co2_tiny", 150), ("co2_triclinic", 300)])
def test_tracks_fp64_engine(cuda, name, n):
    """Same decisions as the FP64 engine, in an orthorhombic and a triclinic
    box (the FP64 pair distance then goes through the box matrix)."""
    c = load(name)
    s = system_of(c)
    mols = np.array(c["molecules"])
    _, a = engine_run(s, mols, n, native.RGPU_FP64, cluster=2)
    _, b = engine_run(s, mols, n, native.RGPU_MIXED_CC64, cluster=2)
    assert a["counters"][4:8].sum() > 10
    np.testing.assert_array_equal(a["counters"][:9], b["counters"][:9])
    kT = units.K_B * s.temperature
    np.testing.assert_allclose(b["energy"][:6], a["energy"][:6], rtol=1e-5, atol=1e-3 * kT)
    # the real-space charge-charge sums (host, adsorbate) in FP64: closer
    # than the FP32 LJ terms
    np.testing.assert_allclose(b["energy"][[2, 3]], a["energy"][[2, 3]], rtol=1e-7, atol=1e-4 * kT)


def drift_run(s, mols, precision, n, threads, cluster, seed=99):
    g = native.GpuSystem(s, maxmol=256, seed=seed, stream_id=1)
    g.set_adsorbates(mols)
    g.set_energy(np.concatenate([g.total_energy(), [0, 0]]))
    eng = native.Engine([g], precision=precision, threads=threads, cluster=cluster)
    eng.run(n)
    eng.sync()
    st = g.state()
    assert st["status"] == 0
    e1 = g.total_energy()
    kT = units.K_B * s.temperature
    eng.close()
    return (np.asarray(st["energy"][:6]) - e1) / kT, int(st["counters"][4:8].sum()), e1 / kT


@pytest.mark.parametrize("threads,cluster", [(256, 2), (1024, 1)])
def test_drift_below_mixed(cuda, threads, cluster):
    """co2_config1 (1536 charged framework atoms) from 4 molecules: after
    3000 moves the real-space and Fourier terms of the CC64 engine are within
    1e-6 k_B T per accepted move of the recomputation, and its total error is
    below the mixed engine's on the same run and below 1e-7 relative."""
    c = load("co2_config1")
    s = system_of(c)
    mols = np.array(c["molecules"])[:4]
    d_mix, acc_mix, _ = drift_run(s, mols, native.RGPU_MIXED, 3000, threads, cluster)
    d_cc, acc_cc, e1 = drift_run(s, mols, native.RGPU_MIXED_CC64, 3000, threads, cluster)
    assert acc_cc > 100 and acc_mix > 100
    assert np.all(np.abs(d_cc[2:6]) <= 1e-6 * acc_cc), d_cc
    assert abs(d_cc.sum()) < abs(d_mix.sum()), (d_cc, d_mix)
    assert abs(d_cc.sum()) <= 1e-7 * abs(e1.sum()), (d_cc.sum(), e1.sum())


def test_refuses_flexible_and_grid_systems(cuda):
    s = systems.hexane_system(n_atoms=512, cell=24.0)
    g = native.GpuSystem(s, maxmol=8, seed=1)
    g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
    with pytest.raises(RuntimeError):
        native.Engine([g], precision=native.RGPU_MIXED_CC64, threads=256, cluster=1)
