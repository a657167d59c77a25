"""Batched state transfer of an engine's systems (rgpu_engine_get_state,
rgpu_engine_set_adsorbates): the same values as the per-system calls, and a
batch uploaded in one transfer continues the same trajectories as one
uploaded system by system."""
import numpy as np
import pytest

from raspa2_b200 import native, systems

pytestmark = pytest.mark.gpu

CLOCK = [15, 16, 17]     # SM clock-cycle counters: not part of a trajectory


def _fresh(sl, maxmol=256):
    return [native.GpuSystem(s, maxmol=maxmol, seed=11, stream_id=i) for i, s in enumerate(sl)]


def test_get_state_equals_per_system_calls(cuda):
    sl = systems.batched_co2_systems(6, seed=5)
    gs = _fresh(sl)
    for g in gs:
        g.set_adsorbates(np.zeros((0, 3, 3)))
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=512, cluster=2)
    e.run(800)
    e.sync()
    states = e.get_states()
    assert sum(st["nmol"] for st in states) > 0
    for g, st in zip(gs, states):
        ref = g.state()
        np.testing.assert_array_equal(st["energy"], ref["energy"])
        np.testing.assert_array_equal(st["counters"], ref["counters"])
        assert (st["nmol"], st["status"], st["step"]) == (ref["nmol"], ref["status"], ref["step"])
        np.testing.assert_array_equal(st["xyz"], g.adsorbates()[: st["nmol"]])


def test_batched_upload_continues_the_same_trajectories(cuda):
    sl = systems.batched_co2_systems(6, seed=5)
    gs = _fresh(sl)
    for g in gs:
        g.set_adsorbates(np.zeros((0, 3, 3)))
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=512, cluster=2)
    e.run(600)
    e.sync()
    xs = [st["xyz"].copy() for st in e.get_states()]
    # the views of one call are overwritten by the next, with the same values here
    again = e.get_states()
    assert all(np.array_equal(a["xyz"], x) for a, x in zip(again, xs))
    runs = []
    for batched in (False, True):
        hs = _fresh(sl)
        eng = native.Engine(hs, precision=native.RGPU_MIXED, threads=512, cluster=2)
        if batched:
            eng.set_adsorbates(xs)
        else:
            for h, x in zip(hs, xs):
                h.set_adsorbates(x)
        eng.run(500)
        eng.sync()
        runs.append([dict(st, xyz=st["xyz"].copy()) for st in eng.get_states()])
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a["energy"], b["energy"])
        np.testing.assert_array_equal(np.delete(a["counters"], CLOCK), np.delete(b["counters"], CLOCK))
        np.testing.assert_array_equal(a["xyz"], b["xyz"])


def test_batched_upload_rejects_overfull_system(cuda):
    sl = systems.batched_co2_systems(2, seed=5)
    gs = _fresh(sl, maxmol=2)
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=512, cluster=2)
    with pytest.raises(native.NativeError):
        e.set_adsorbates([np.zeros((3, 3, 3)), np.zeros((0, 3, 3))])
