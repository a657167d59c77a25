"""A triclinic box (cell angles 80, 95, 110 degrees; the CO2 model of
config 1): the reference's triclinic minimum image, wave vectors and random
positions on the GPU.

- The per-call entry points against the reference's own outputs for this
  box are in tests/test_gpu_parity.py (case co2_triclinic).
- The FP64 engine follows the oracle's GCMC trajectory move for move (the
  oracle is pinned to the reference for this box by
  tests/test_oracle_golden.py).
- The mixed engine's running energies equal an FP64 recomputation.
- Energy grids are refused in a triclinic box.
"""
import numpy as np
import pytest

from raspa2_b200 import native, units

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


def test_grids_are_refused(cuda):
    import torch
    s = system_of(load("co2_triclinic"))
    g = native.GpuSystem(s, maxmol=8)
    buf = torch.zeros(16 * 16 * 16 * 8, dtype=torch.float32, device="cuda")
    with pytest.raises(native.NativeError, match="triclinic"):
        g.grid_build(0, [15, 15, 15], list(s.box), [0, 0, 0], buf.data_ptr())
