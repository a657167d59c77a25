"""The persistent batched engine against the oracle's GCMC on the same
counter-based random stream, plus energy-drift and batching checks."""
import numpy as np
import pytest

from oracle import oracle as O
from raspa2_b200 import native, systems, units

from golden_cases import load, system_of

pytestmark = pytest.mark.gpu


def engine_run(sysm, mols, nsteps, precision, seed=777, stream_id=3, threads=256, maxmol=64, cluster=0,
               ctas_per_sm=1):
    g = native.GpuSystem(sysm, maxmol=maxmol, seed=seed, stream_id=stream_id)
    g.set_adsorbates(mols)
    e = native.Engine([g], precision=precision, threads=threads, cluster=cluster, ctas_per_sm=ctas_per_sm)
    e.run(nsteps)
    e.sync()
    return g, g.state()


def oracle_run(sysm, mols, nsteps, seed=777, stream_id=3, maxmol=64):
    o = O.Oracle.from_system(sysm, maxmol=maxmol)
    o.set_molecules(mols)
    p = O.mc_params(sysm, seed, stream_id)
    st = O.MCState()
    o.mc_run(p, st, 0, nsteps)
    return o, st


@pytest.mark.parametrize("name,cluster,occ", [("co2_tiny", 1, 1), ("co2_tiny", 2, 1), ("co2_config1", 8, 1),
                                              ("co2_config1", 3, 1), ("methane_config0", 2, 1),
                                              ("co2_config1", 2, 2)])
def test_fp64_engine_reproduces_oracle_trajectory(cuda, name, cluster, occ):
    """Same counter-based stream, same decisions: the FP64 engine (framework
    split over `cluster` CTAs; with occ = 2 sized for two CTAs per SM, so
    with less staged in shared memory) follows the oracle's GCMC trajectory."""
    c = load(name)
    s = system_of(c)
    mols = np.array(c["molecules"])
    n = 300
    g, st = engine_run(s, mols, n, native.RGPU_FP64, cluster=cluster, ctas_per_sm=occ)
    o, ost = oracle_run(s, mols, n)
    assert st["status"] == 0
    assert st["step"] == n
    np.testing.assert_array_equal(st["counters"][0:4], np.array(ost.attempts[:4]))
    np.testing.assert_array_equal(st["counters"][4:8], np.array(ost.accepted[:4]))
    assert st["counters"][8] == ost.moves
    assert st["nmol"] == o.nmol
    np.testing.assert_allclose(g.adsorbates(), o.molecules(), rtol=0, atol=1e-10)
    # running energy changes (engine order: hv, av, hc, ac, hF, aF)
    np.testing.assert_allclose(st["energy"][:6], np.array(ost.u), rtol=1e-9, atol=1e-6)


@pytest.mark.parametrize("name,cluster", [("co2_tiny", 1), ("co2_tiny", 2), ("methane_config0", 2)])
def test_fp64_engine_reinsertion_and_widom_follow_oracle(cuda, name, cluster):
    """All six move types, CBMC reinsertion and Widom test insertions
    included: the FP64 engine follows the oracle's trajectory, and the Widom
    Rosenbluth-weight sums agree."""
    import dataclasses
    c = load(name)
    s = system_of(c)
    s = dataclasses.replace(s, moves=systems.MoveMix(translation=1.0, rotation=1.0 if s.molecule.n_atoms > 1 else 0.0,
                                                     swap_insert=0.5, swap_delete=0.5, reinsertion=1.0, widom=1.0))
    mols = np.array(c["molecules"])
    n = 400
    g, st = engine_run(s, mols, n, native.RGPU_FP64, cluster=cluster)
    o, ost = oracle_run(s, mols, n)
    assert st["status"] == 0
    np.testing.assert_array_equal(st["counters"][0:4], np.array(ost.attempts[:4]))
    np.testing.assert_array_equal(st["counters"][4:8], np.array(ost.accepted[:4]))
    assert st["counters"][18] == ost.attempts[4] > 0
    assert st["counters"][19] == ost.accepted[4]
    assert st["counters"][8] == ost.moves
    assert st["nmol"] == o.nmol
    np.testing.assert_allclose(g.adsorbates(), o.molecules(), rtol=0, atol=1e-10)
    np.testing.assert_allclose(st["energy"][:6], np.array(ost.u), rtol=1e-9, atol=1e-6)
    sums = g.averages()["sums"]
    assert sums[7] == ost.widom_n > 0
    np.testing.assert_allclose(sums[6], ost.widom_sum, rtol=1e-9, atol=1e-300)


@pytest.mark.parametrize("precision,tol,cluster", [(native.RGPU_FP64, 1e-10, 2), (native.RGPU_MIXED, 1e-6, 2),
                                                   (native.RGPU_MIXED, 1e-6, 1)])
def test_energy_drift(cuda, precision, tol, cluster):
    """Running totals after many accepted moves equal a full recomputation
    (the reference's energy-drift check, src/output.c:7032)."""
    c = load("co2_config1")
    s = system_of(c)
    g = native.GpuSystem(s, maxmol=128, seed=99, stream_id=1)
    g.set_adsorbates(np.array(c["molecules"])[:4])
    e0 = g.total_energy()
    g.set_energy(np.concatenate([e0, [0, 0]]))
    eng = native.Engine([g], precision=precision, cluster=cluster)
    eng.run(2000)
    eng.sync()
    st = g.state()
    assert st["status"] == 0
    acc = st["counters"][4:8].sum()
    assert acc > 20
    e1 = g.total_energy()
    kT = units.K_B * s.temperature
    drift = np.abs(st["energy"][:6] - e1)
    scale = np.maximum(np.abs(e1), kT)
    assert np.all(drift <= tol * scale * max(1.0, acc / 100.0)), (st["energy"][:6], e1, drift / scale)


def test_batched_systems_match_single_runs(cuda):
    """Each system's result is bitwise the same alone and in a batch of
    uneven systems at the same launch shape (independent random streams, one
    cluster per system)."""
    specs = [systems.tiny_co2_system(seed=7), systems.co2_system(seed=21, n_atoms=512, cell=20.0, kmax=5),
             systems.methane_system(seed=3)]
    n = 200
    alone = []
    for i, s in enumerate(specs):
        g, st = engine_run(s, np.zeros((0, s.molecule.n_atoms, 3)), n, native.RGPU_MIXED, seed=5, stream_id=i)
        alone.append((st, g.adsorbates()))
    gs = []
    for i, s in enumerate(specs):
        g = native.GpuSystem(s, maxmol=64, seed=5, stream_id=i)
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
        gs.append(g)
    # same launch shape as engine_run (the unit split, hence the FP32
    # summation order, follows the CTA size)
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=256)
    e.run(n)
    e.sync()
    for g, (st, xyz) in zip(gs, alone):
        st2 = g.state()
        # counters 15.. are SM clock cycles (timing, not results)
        np.testing.assert_array_equal(st2["counters"][:15], st["counters"][:15])
        assert st2["nmol"] == st["nmol"]
        np.testing.assert_array_equal(st2["energy"], st["energy"])
        np.testing.assert_array_equal(g.adsorbates(), xyz)


def test_mixed_engine_tracks_fp64(cuda):
    """Same random stream: the mixed engine takes the same decisions as the
    FP64 engine over a short run (decisions are FP64 on FP32-accurate sums)."""
    c = load("co2_tiny")
    s = system_of(c)
    mols = np.array(c["molecules"])
    _, a = engine_run(s, mols, 150, native.RGPU_FP64, cluster=2)
    _, b = engine_run(s, mols, 150, native.RGPU_MIXED, cluster=2)
    np.testing.assert_array_equal(a["counters"][:9], b["counters"][:9])
    kT = units.K_B * s.temperature
    np.testing.assert_allclose(b["energy"][:6], a["energy"][:6], rtol=1e-5, atol=1e-3 * kT)


def test_autotune_leaves_systems_untouched(cuda):
    """The tuner times shapes on copies: the caller's systems keep their
    configuration, counters and random-stream position."""
    from raspa2_b200 import autotune
    specs = [systems.tiny_co2_system(seed=7), systems.tiny_co2_system(seed=8)]
    gs = []
    for i, s in enumerate(specs):
        g = native.GpuSystem(s, maxmol=64, seed=5, stream_id=i)
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
        gs.append(g)
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=256, cluster=1)
    e.run(200)
    e.sync()
    before = [(g.adsorbates().copy(), g.state()) for g in gs]
    shape = autotune.tune(gs, precision=native.RGPU_MIXED, moves=50, warm=10, shapes=[(1, 256), (2, 256)],
                          use_cache=False)
    assert (shape.cluster, shape.threads) in [(1, 256), (2, 256)]
    assert all("moves_per_s" in row for row in shape.table)
    for g, (xyz, st) in zip(gs, before):
        np.testing.assert_array_equal(g.adsorbates(), xyz)
        st2 = g.state()
        np.testing.assert_array_equal(st2["counters"][:15], st["counters"][:15])
        assert st2["step"] == st["step"]


def test_graph_replay_matches_direct_launches(cuda):
    """rgpu_engine_use_graph: replaying the captured launch advances the
    systems exactly as direct launches do."""
    s = systems.tiny_co2_system(seed=7)
    out = []
    for graph in (False, True):
        g = native.GpuSystem(s, maxmol=64, seed=9, stream_id=2)
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
        e = native.Engine([g], precision=native.RGPU_MIXED, threads=256, cluster=2)
        e.use_graph(graph)
        for _ in range(3):
            e.run(150)
        e.run(40)          # a different step count is captured anew
        e.sync()
        out.append((g.state(), g.adsorbates()))
    (a, xa), (b, xb) = out
    assert a["step"] == b["step"] == 490
    np.testing.assert_array_equal(a["counters"][:15], b["counters"][:15])
    np.testing.assert_array_equal(a["energy"], b["energy"])
    np.testing.assert_array_equal(xa, xb)


def test_split_launch_matches_single_runs(cuda):
    """rgpu_engine_set_split: the systems moved to a second launch at cluster
    3 run bitwise as they do alone at cluster 3, the others as alone at
    cluster 1, also when the two launches are replayed from one CUDA graph;
    the batched state read (device slots reordered) returns each system's
    own state, and a batched upload reaches the right systems."""
    specs = [systems.tiny_co2_system(seed=7), systems.co2_system(seed=21, n_atoms=512, cell=20.0, kmax=5),
             systems.methane_system(seed=3)]
    second = [2, 0]
    n = 200
    alone = []
    for i, s in enumerate(specs):
        g, st = engine_run(s, np.zeros((0, s.molecule.n_atoms, 3)), n, native.RGPU_MIXED, seed=5, stream_id=i,
                           cluster=3 if i in second else 1)
        alone.append((st, g.adsorbates()))
    gs = []
    for i, s in enumerate(specs):
        g = native.GpuSystem(s, maxmol=64, seed=5, stream_id=i)
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
        gs.append(g)
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=256, cluster=1)
    e.set_split(second, 3)
    e.use_graph(True)
    e.run(n)
    e.sync()
    batched = e.get_states()
    for g, b, (st, xyz) in zip(gs, batched, alone):
        st2 = g.state()
        np.testing.assert_array_equal(st2["counters"][:15], st["counters"][:15])
        assert st2["nmol"] == st["nmol"] and b["nmol"] == st["nmol"]
        np.testing.assert_array_equal(st2["energy"], st["energy"])
        np.testing.assert_array_equal(b["energy"], st["energy"])
        np.testing.assert_array_equal(b["counters"][:15], st["counters"][:15])
        np.testing.assert_array_equal(g.adsorbates(), xyz)
        np.testing.assert_array_equal(b["xyz"], xyz)
    # a batched upload lands in each system's own slot
    e.set_adsorbates([xyz[: max(len(xyz) - 1, 0)] for _, xyz in alone])
    for g, (_, xyz) in zip(gs, alone):
        np.testing.assert_array_equal(g.adsorbates(), xyz[: max(len(xyz) - 1, 0)])
    with pytest.raises(native.NativeError):
        e.set_split([0, 1, 2], 2)
    with pytest.raises(native.NativeError):
        e.set_split([1, 1], 2)
    e.set_split([], 0)
    e.run(10)
    e.sync()
    assert all(g.state()["status"] == 0 for g in gs)


def test_mixed_running_totals_within_1e6_on_batched_boxes(cuda):
    """The metric's bound on its own workload: the first 8 boxes of the
    batched CO2 set (512-4096 framework atoms per cell, charges up to
    +-1.2 e), grown from empty over 2000 moves each in one mixed engine;
    every box's running total energy is within 1e-6 relative of an FP64
    recomputation of its final configuration."""
    specs = systems.batched_co2_systems(64, seed=2)[:8]
    gs = []
    for i, s in enumerate(specs):
        g = native.GpuSystem(s, maxmol=768, seed=20240, stream_id=i)
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
        gs.append(g)
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=512, cluster=2)
    for _ in range(4):
        e.run(500)
    e.sync()
    worst = 0.0
    for g in gs:
        st = g.state()
        assert st["status"] == 0
        if st["nmol"] == 0:
            continue
        ref = np.asarray(g.total_energy())
        worst = max(worst, abs(np.sum(st["energy"][:6]) - ref.sum()) / abs(ref.sum()))
    assert worst <= 1e-6, worst
