"""The continuous-batching server: every job's result is bitwise the same
alone and in a mix of jobs admitted at different times (per-job random
streams, engine step limits, fixed launch shape), and admission respects the
device-memory budget."""
import dataclasses

import numpy as np
import pytest

from raspa2_b200 import native, serve, systems

pytestmark = pytest.mark.gpu


def _jobs():
    co2 = systems.tiny_co2_system(seed=7)
    ch4 = systems.methane_like_system(seed=4, n_atoms=600)
    specs = [(co2, 1e5, 298.0, 1400), (ch4, 1e6, 300.0, 900), (dataclasses.replace(co2, name="co2b"), 1e6, 323.0, 700),
             (ch4, 1e4, 273.0, 1100)]
    jobs = []
    for i, (s, p, T, n) in enumerate(specs):
        s = dataclasses.replace(s, pressure=p, temperature=T)
        jobs.append(serve.Job(id=i, system=s, steps=n, equil=n // 3, seed=50 + i, arrival=0.0, maxmol=64))
    return jobs


def _fresh(jobs, arrivals=None):
    out = []
    for k, j in enumerate(jobs):
        out.append(serve.Job(id=j.id, system=j.system, steps=j.steps, equil=j.equil, seed=j.seed,
                             arrival=0.0 if arrivals is None else arrivals[k], maxmol=j.maxmol))
    return out


def _same(a, b):
    for key in ("loading", "energy_K", "samples", "final_nmol", "steps", "energy_terms", "counters"):
        assert a[key] == b[key], (key, a[key], b[key])


def test_result_same_alone_and_in_mix(cuda):
    base = _jobs()
    alone = []
    for j in _fresh(base):
        serve.Server(chunk=200, threads=256).run([j], realtime=False)
        alone.append(j.result)
    # the mix: all jobs together, and a second mix where two arrive late
    # (admitted at later launch boundaries, next to jobs already running)
    mixed = _fresh(base)
    st = serve.Server(chunk=200, threads=256).run(mixed, realtime=False)
    assert st["max_active"] == len(base)
    late = _fresh(base, arrivals=[0.0, 0.0, 0.05, 0.1])
    serve.Server(chunk=200, threads=256).run(late, realtime=True)
    for a, m, l in zip(alone, mixed, late):
        assert a["steps"] == m.result["steps"] == l.result["steps"]
        _same(a, m.result)
        _same(a, l.result)
        assert a["samples"] == m.steps - m.equil


def test_memory_budget_limits_admission(cuda):
    jobs = _fresh(_jobs())
    fp = sorted(serve.footprint_bytes(j) for j in jobs)
    # no two jobs fit together; a job is admitted alone even above the budget
    budget = fp[0] + fp[1] - 1
    st = serve.Server(chunk=300, threads=256, mem_budget=budget).run(jobs, realtime=False)
    assert st["max_active"] == 1
    assert all(j.result is not None and j.result["steps"] == j.steps for j in jobs)
    assert st["p99_job_ms"] >= st["p50_job_ms"] > 0


def test_served_job_returns_raspa_output(cuda):
    """A job with raspa_output returns its production as five equal blocks
    (the job pauses at each boundary) and the `.data` results text; the
    blocks add up to the job's own averages, and the reference's parser
    layout is produced (tests/test_restart_output.py checks the parser)."""
    from raspa2_b200 import output
    s = dataclasses.replace(systems.tiny_co2_system(seed=7), pressure=1e6, temperature=298.0)
    job = serve.Job(id=5, system=s, steps=2400, equil=400, seed=31, maxmol=64, raspa_output=True)
    plain = serve.Job(id=5, system=s, steps=2400, equil=400, seed=31, maxmol=64)
    serve.Server(chunk=300, threads=256).run([job], realtime=False)
    serve.Server(chunk=300, threads=256).run([plain], realtime=False)
    r = job.result
    assert r["steps"] == 2400 and len(r["blocks"]) == output.NR_BLOCKS
    assert [b.samples for b in r["blocks"]] == [400.0] * output.NR_BLOCKS
    # pausing at the block boundaries leaves the trajectory unchanged; the
    # energy sum is added up over other launches, so it may differ in the
    # last bits
    for key in ("loading", "samples", "final_nmol", "energy_terms", "counters"):
        assert r[key] == plain.result[key], key
    assert abs(r["energy_K"] - plain.result["energy_K"]) <= 1e-12 * abs(plain.result["energy_K"])
    n = sum(b.n for b in r["blocks"]) / sum(b.samples for b in r["blocks"])
    assert abs(n - r["loading"]) <= 1e-12 * max(1.0, n)
    assert "Average loading absolute [molecules/unit cell]" in r["raspa_summary"]
    assert "Enthalpy of adsorption:" in r["raspa_summary"]


def test_jobs_reuse_the_slots_of_finished_ones(cuda):
    """With two slots, later jobs go into the slots of finished ones
    (rgpu_engine_replace_system, a system of another framework and size in
    place of the old one) and their results are bitwise those of the jobs run
    alone."""
    base = _jobs()
    alone = []
    for j in _fresh(base):
        serve.Server(chunk=200, threads=256).run([j], realtime=False)
        alone.append(j.result)
    jobs = _fresh(base)
    st = serve.Server(chunk=200, threads=256, max_slots=2).run(jobs, realtime=False)
    assert st["max_active"] == 2 and st["slot_replacements"] >= 1
    for a, j in zip(alone, jobs):
        _same(a, j.result)


def test_engine_outlives_a_replaced_and_destroyed_system(cuda):
    """The engine keeps no resource of a system it no longer holds: slot 0's
    system replaced, then destroyed, and the engine runs on."""
    a = native.GpuSystem(systems.tiny_co2_system(seed=7), maxmol=16, seed=1, stream_id=0)
    b = native.GpuSystem(systems.tiny_co2_system(seed=8), maxmol=16, seed=2, stream_id=1)
    c = native.GpuSystem(systems.tiny_co2_system(seed=9), maxmol=16, seed=3, stream_id=2)
    eng = native.Engine([a, b], precision=native.RGPU_MIXED, threads=256, cluster=1)
    eng.run(50)
    eng.sync()
    assert eng.replace(0, c)
    a.close()
    eng.run(50)
    eng.sync()
    st = c.state()
    assert st["status"] == 0 and int(st["step"]) == 50
    assert int(b.state()["step"]) == 100
    eng.close()
    np.testing.assert_array_equal(c.state()["counters"], st["counters"])
