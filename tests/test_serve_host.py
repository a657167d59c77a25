"""The serving loop's host logic on CPU: admission on its own thread, slots
reused in place, the memory budget and the step accounting, with the
library and the CUDA runtime replaced by fakes that advance each system by
the engine's rule (a launch takes every system in a slot `chunk` steps on,
but not past its step limit)."""
import dataclasses
import threading
import types

import numpy as np
import pytest

from raspa2_b200 import native, serve, systems


class FakeSystem:
    live = 0
    lock = threading.Lock()

    def __init__(self, sysm, maxmol=512, seed=1, stream_id=0):
        self.sysm, self.maxmol, self.seed, self.stream_id = sysm, maxmol, seed, stream_id
        self.step, self.limit, self.closed = 0, 0, False
        with FakeSystem.lock:
            FakeSystem.live += 1

    def set_adsorbates(self, xyz):
        pass

    def set_limits(self, end_step, avg_start=0):
        self.limit = end_step

    def state(self):
        return {"step": self.step, "nmol": 0, "status": 0, "energy": np.zeros(8), "counters": np.zeros(20)}

    def averages(self):
        return {"loading": 0.0, "energy": 0.0, "enthalpy": float("nan"), "samples": self.step, "sums": np.zeros(8)}

    def close(self):
        assert not self.closed, "system closed twice"
        self.closed = True
        with FakeSystem.lock:
            FakeSystem.live -= 1


class FakeEngine:
    def __init__(self, systems_, precision=0, threads=0, cluster=1):
        assert not any(g.closed for g in systems_)
        self.systems = list(systems_)

    def use_graph(self, on):
        pass

    def replace(self, i, g, stream=None):
        self.systems[i] = g
        return True

    def run(self, n, stream=None):
        for g in set(self.systems):
            assert not g.closed, "a closed system is still in the engine"
            g.step = min(g.step + n, max(g.limit, g.step))

    def sync(self):
        pass

    def close(self):
        pass


class FakeEvent:
    def __init__(self, enable_timing=False):
        pass

    def record(self, stream=None):
        pass

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return 1.0


@pytest.fixture
def fakes(monkeypatch):
    import torch
    monkeypatch.setattr(native, "GpuSystem", FakeSystem)
    monkeypatch.setattr(native, "Engine", FakeEngine)
    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda d: types.SimpleNamespace(multi_processor_count=6))
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 0)
    monkeypatch.setattr(torch.cuda, "Stream", lambda *a, **k: types.SimpleNamespace(cuda_stream=0))
    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    FakeSystem.live = 0
    yield


def _jobs(n, arrivals=None):
    base = systems.tiny_co2_system()
    out = []
    for i in range(n):
        s = dataclasses.replace(base, name=f"j{i}")
        out.append(serve.Job(id=i, system=s, steps=100 * (1 + i % 5), equil=10, seed=i,
                             arrival=0.0 if arrivals is None else arrivals[i], maxmol=32))
    return out


@pytest.mark.parametrize("realtime", [False, True])
def test_every_job_runs_to_its_step_count(fakes, realtime):
    arrivals = list(np.linspace(0.0, 0.05, 30)) if realtime else None
    jobs = _jobs(30, arrivals)
    st = serve.Server(chunk=40, max_slots=4, lookahead=3).run(jobs, realtime=realtime)
    assert all(j.result is not None and j.result["steps"] == j.steps for j in jobs)
    assert st["mc_steps"] == sum(j.steps for j in jobs)
    assert 1 <= st["max_active"] <= 4
    assert st["engine_builds"] == 1 and 30 - 4 <= st["slot_replacements"] <= 30 - 1
    assert all(j.started >= j.admitted >= j.arrival and j.finished >= j.started for j in jobs)
    assert FakeSystem.live == 0          # every system freed, none twice


def test_memory_budget_holds_one_job_at_a_time(fakes):
    jobs = _jobs(6)
    fp = serve.footprint_bytes(jobs[0])
    st = serve.Server(chunk=50, max_slots=4, lookahead=3, mem_budget=1.5 * fp).run(jobs, realtime=False)
    assert st["max_active"] == 1
    assert all(j.result["steps"] == j.steps for j in jobs)


def test_admission_error_reaches_the_caller(fakes, monkeypatch):
    def bad(self, job, now):
        raise RuntimeError("set-up failed")
    monkeypatch.setattr(serve.Server, "_admit", bad)
    with pytest.raises(RuntimeError, match="set-up failed"):
        serve.Server(chunk=50, max_slots=2).run(_jobs(3), realtime=False)
