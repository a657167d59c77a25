"""Checkpoints and restart files on the GPU path.

- A system restored from a checkpoint continues the saved trajectory move for
  move: positions, running energies, counters and ensemble sums are bitwise
  those of the run that was not interrupted (mixed engine; rigid CO2 with
  Ewald, flexible hexane).
- A checkpoint is refused by a system of another framework or molecule, and
  accepted by one at another pressure.
- A served job resumed from its checkpoint ends with the result of the job
  that ran straight through.
- A restart file written by the reference loads into a GPU system, whose FP64
  energies equal those the reference printed for it.
"""
import dataclasses
import json
import os

import numpy as np
import pytest

from raspa2_b200 import native, restart, serve, systems, units

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CLOCK_COUNTERS = [15, 16, 17]     # SM clock cycles: not part of the trajectory


def _state(g):
    st = g.state()
    c = np.delete(st["counters"], CLOCK_COUNTERS)
    return st["energy"], c, st["nmol"], st["step"], st["status"], g.adsorbates(), g.averages()["sums"]


def _assert_same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(np.asarray(x), np.asarray(y))


CASES = {
    "co2": (lambda: systems.co2_system(seed=1), 256, 2, 512),
    "hexane": (lambda: systems.hexane_system(seed=4, n_atoms=1200, cell=26.0, pressure=1e6), 64, 2, 256),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_checkpoint_resume_is_bitwise(cuda, case):
    build, maxmol, cluster, threads = CASES[case]
    s = build()
    n1, n2 = 1500, 1500
    a = native.GpuSystem(s, maxmol=maxmol, seed=99, stream_id=7)
    a.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
    a.set_limits(0, 500)
    e = native.Engine([a], precision=native.RGPU_MIXED, threads=threads, cluster=cluster)
    e.run(n1)
    e.sync()
    ck = a.checkpoint()
    assert a.state()["nmol"] > 3
    e.run(n2)
    e.sync()
    straight = _state(a)
    e.close()

    b = native.GpuSystem(s, maxmol=maxmol, seed=99, stream_id=7)
    b.restore(ck)
    assert b.state()["step"] == n1
    e2 = native.Engine([b], precision=native.RGPU_MIXED, threads=threads, cluster=cluster)
    e2.run(n2)
    e2.sync()
    _assert_same(straight, _state(b))


def test_checkpoint_refused_by_another_model(cuda):
    s = systems.co2_system(seed=1)
    a = native.GpuSystem(s, maxmol=64, seed=1)
    a.set_adsorbates(np.zeros((0, 3, 3)))
    e = native.Engine([a], precision=native.RGPU_MIXED, threads=512, cluster=2)
    e.run(300)
    e.sync()
    ck = a.checkpoint()
    other = native.GpuSystem(systems.co2_system(seed=2), maxmol=64, seed=1)
    with pytest.raises(native.NativeError):
        other.restore(ck)
    ch4 = native.GpuSystem(systems.methane_system(seed=0), maxmol=64, seed=1)
    with pytest.raises(native.NativeError):
        ch4.restore(ck)
    with pytest.raises(native.NativeError):
        a.restore(ck[:-8])
    small = native.GpuSystem(s, maxmol=1, seed=1)
    if a.state()["nmol"] > 1:
        with pytest.raises(native.NativeError):
            small.restore(ck)
    # another state point of the same model: accepted, same molecules
    hp = native.GpuSystem(dataclasses.replace(s, pressure=1e7), maxmol=64, seed=5)
    hp.restore(ck)
    np.testing.assert_array_equal(hp.adsorbates(), a.adsorbates())


def test_served_job_resumes_from_checkpoint(cuda):
    s = dataclasses.replace(systems.tiny_co2_system(seed=7), pressure=1e6, temperature=298.0)
    full = serve.Job(id=3, system=s, steps=1600, equil=400, seed=21, maxmol=64)
    serve.Server(chunk=200, threads=256).run([full], realtime=False)
    half = serve.Job(id=3, system=s, steps=800, equil=400, seed=21, maxmol=64, keep_checkpoint=True)
    serve.Server(chunk=200, threads=256).run([half], realtime=False)
    rest = serve.Job(id=3, system=s, steps=1600, equil=400, seed=21, maxmol=64, resume=half.result["checkpoint"])
    serve.Server(chunk=200, threads=256).run([rest], realtime=False)
    for key in ("loading", "energy_K", "samples", "final_nmol", "steps", "energy_terms", "counters"):
        assert full.result[key] == rest.result[key], key


@pytest.mark.parametrize("name,build", [("co2_config1", lambda: systems.co2_system(seed=1)),
                                        ("hexane_small", lambda: systems.hexane_system(seed=4, n_atoms=1200,
                                                                                       cell=26.0))])
def test_reference_restart_file_on_gpu(cuda, name, build):
    meta = json.load(open(os.path.join(GOLDEN, f"restart_{name}.json")))
    s = dataclasses.replace(build(), pressure=meta["pressure_Pa"], temperature=meta["temperature_K"])
    xyz = restart.read_restart(os.path.join(GOLDEN, f"restart_{name}.txt")).component(s.molecule.name).positions
    g = native.GpuSystem(s, maxmol=len(xyz) + 8, seed=1)
    g.set_adsorbates(xyz)
    u = g.total_energy() * units.ENERGY_TO_KELVIN
    ref = meta["energies_K"]
    keys = ["Host/Adsorbate VDW energy", "Adsorbate/Adsorbate VDW energy", "Host/Adsorbate charge-charge Real energy",
            "Adsorbate/Adsorbate charge-charge Real energy", "Host/Adsorbate charge-charge Fourier energy",
            "Adsorbate/Adsorbate charge-charge Fourier energy"]
    for k, v in zip(keys, u):
        assert abs(v - ref[k]) <= 1e-9 * abs(ref[k]) + 2e-8, (k, v, ref[k])
    if not s.molecule.rigid:
        intra = g.intra_energy() * units.ENERGY_TO_KELVIN
        r = ref["Adsorbate bend energy"] + ref["Adsorbate torsion energy"] + ref["Adsorbate intra VDW energy"]
        assert abs(intra - r) <= 1e-9 * abs(r) + 2e-8
