"""Continuous-batching server of isotherm-point GCMC jobs on one GPU.

A job is one adsorption state point: a framework, an adsorbate, a temperature
and a pressure, run for a number of MC steps. The first `equil` steps
equilibrate the loading; the steps after them are sampled.

The server keeps every admitted job's state on the device until the job
ends: positions, S(k) and the running energies. It advances all admitted
jobs together, one engine launch of `chunk` MC steps at a time, so
`chunk` is the granularity at which jobs are admitted and retired. Between
launches:

- jobs whose step count is reached are retired, and their averages are read
  back;
- jobs that have arrived are admitted, as long as both hold:
  - an engine slot is free (one cluster per job; slots = SMs / cluster
    size), or will be: up to `lookahead` jobs beyond the slots are admitted
    ahead and wait, set up, for the next free slot;
  - the job's estimated device-memory footprint fits the budget.

A newly admitted job's device set-up (framework upload, structure factors)
runs on a host thread of its own and on the job system's own stream, while
the serving loop launches and retires, so admission overlaps the other jobs'
work on the GPU; a job admitted ahead goes into the slot of a finished one
at the next launch without set-up work in between.

The engine stops each job exactly at its step count (rgpu_system_set_limits).
Each job has its own random stream, and the launch shape is fixed for the
server's lifetime. A job's result is therefore bitwise the same whether it
runs alone or in a mix, whatever else is admitted beside it.

This is the host-side request loop; all MC work runs in the engine kernel.
"""
from __future__ import annotations

import collections
import dataclasses
import gc
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import native, output, ranks, systems, units

# a reference cycle is max(MinimumInnerCycles = 20, N) MC steps
# (src/monte_carlo.c:367, src/input.c:346)
RASPA_MIN_STEPS_PER_CYCLE = 20


@dataclasses.dataclass
class Job:
    id: int
    system: systems.System
    steps: int                  # MC steps to run
    equil: int = 0              # steps before sampling starts
    seed: int = 1
    arrival: float = 0.0        # seconds after the stream starts
    maxmol: int = 512
    # resumable jobs: start from a checkpoint of the same system and stream
    # (GpuSystem.checkpoint; `steps` and `equil` count from step 0 of the
    # original job), and/or return the final checkpoint with the result
    resume: Optional[bytes] = None
    keep_checkpoint: bool = False
    # RASPA-style results: the production in NR_BLOCKS equal blocks, each
    # block's ensemble sums, and the `.data` results text built from them
    # (raspa2_b200.output); the job pauses at each block boundary until the
    # next launch
    raspa_output: bool = False
    # filled in by the server
    admitted: Optional[float] = None
    started: Optional[float] = None     # placed in an engine slot
    finished: Optional[float] = None
    result: Optional[dict] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def footprint_bytes(job: Job) -> int:
    """Device memory of one job (system_footprint_bytes)."""
    return system_footprint_bytes(job.system, job.maxmol)


def system_footprint_bytes(s: systems.System, maxmol: int) -> int:
    """Device memory of one system as rgpu_system_create allocates it, plus
    the engine's per-system descriptor."""
    nfw = s.n_framework()
    ntile = (nfw + 31) // 32 + 8
    nk = len(systems.kvector_indices(s.kmax)) if s.ewald else 1
    nads = maxmol * s.molecule.n_atoms
    io_n = max(64, nfw, nads)
    b = nfw * 32 + ntile * (32 * 16 + 32)          # fw64, fw32, tiles
    b += nk * (4 + 8 + 16 * 3)                     # kvec, kfactor, S_fw, S_ads, dS
    b += nads * (24 + 16 + 32)                     # positions, records
    b += io_n * 32 + 64 * (32 + 12) + 4096         # per-call scratch, descriptor, state
    return int(b)


def work_estimate(job: Job) -> float:
    """Relative device work of a job: MC steps times the pairs a step
    visits (framework atoms plus, with charges, the wave vectors)."""
    s = job.system
    nk = len(systems.kvector_indices(s.kmax)) if s.ewald else 0
    return float(job.steps) * (s.n_framework() + nk) * s.molecule.n_atoms


def serve_placed(jobs: Sequence[Job], rank: int, world: int, make_server=None, mem_budget: float = 150e9,
                 realtime: bool = True):
    """Serves one job list over `world` GPUs, one server per rank: the jobs
    are placed by device-memory footprint (ranks.place, the same placement
    on every rank, no communication), rank `rank` serves its share with its
    own server, and the per-job results are gathered on rank 0. Returns
    (this rank's job indices, this rank's server statistics, on rank 0 the
    results of all jobs by job id, else None). A job's result does not
    depend on where it runs: each job has its own random stream."""
    parts = ranks.place([footprint_bytes(j) for j in jobs], [work_estimate(j) for j in jobs], world,
                        budget=mem_budget)
    mine = [jobs[i] for i in parts[rank]]
    srv = make_server() if make_server else Server(mem_budget=mem_budget)
    stats = srv.run(mine, realtime=realtime) if mine else {"jobs": 0}
    gathered = ranks.gather_results({j.id: j.result for j in mine})
    allres = None
    if gathered is not None:
        allres = {}
        for d in gathered:
            allres.update(d)
    return parts[rank], stats, allres


class Server:
    """Admits, advances and retires jobs; see the module docstring."""

    def __init__(self, precision: int = native.RGPU_MIXED, threads: int = 1024, cluster: int = 1,
                 chunk: int = 400, max_slots: Optional[int] = None, mem_budget: float = 150e9,
                 lookahead: int = 16):
        import torch

        self.precision = precision
        self.threads = threads
        self.cluster = cluster
        self.chunk = chunk
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        self.max_slots = max_slots or max(1, sms // cluster)
        self.lookahead = lookahead
        self.mem_budget = mem_budget
        self.stream = torch.cuda.Stream()
        self.launches = 0

    def _placeholder(self, jobs: Sequence[Job]) -> Optional["native.GpuSystem"]:
        """A system that takes no step (one step run, limit 1) and holds the
        engine's free slots. It is the job list's largest framework with the
        largest wave-vector set and molecule capacity of the list, so that an
        engine sized with it takes every job of the list in place."""
        if not jobs:
            return None
        big = max(jobs, key=lambda j: j.system.n_framework())
        ew = [j for j in jobs if j.system.ewald]
        s = big.system
        if ew:
            kmax = max((tuple(j.system.kmax) for j in ew), key=lambda k: max(k))
            src = max(ew, key=lambda j: j.system.n_framework()).system
            s = dataclasses.replace(src, kmax=kmax, name="placeholder")
        natom = s.molecule.n_atoms
        maxmol = max((j.maxmol * j.system.molecule.n_atoms + natom - 1) // natom for j in jobs)
        g = native.GpuSystem(s, maxmol=maxmol, seed=1, stream_id=1 << 30)
        g.set_adsorbates(np.zeros((0, natom, 3)))
        g.set_limits(1, 1)
        e = native.Engine([g], precision=self.precision, threads=self.threads, cluster=self.cluster)
        e.run(1, self.stream.cuda_stream)
        e.sync()
        e.close()
        return g

    def _admit(self, job: Job, now: float) -> "native.GpuSystem":
        g = native.GpuSystem(job.system, maxmol=job.maxmol, seed=job.seed, stream_id=job.id)
        if job.resume is not None:
            g.restore(job.resume)
        else:
            g.set_adsorbates(np.zeros((0, job.system.molecule.n_atoms, 3)))
        if job.raspa_output:
            if job.resume is not None and int(g.state()["step"]) > job.equil:
                raise ValueError("raspa_output: the job's production must start within one admission")
            prod = job.steps - job.equil
            job._bounds = [job.equil + prod * (b + 1) // output.NR_BLOCKS for b in range(output.NR_BLOCKS)]
            job._blocks = []
            job._prev = output.Block.from_sums(g.averages()["sums"])
            g.set_limits(self._next_bound(job, int(g.state()["step"])), job.equil)
        else:
            g.set_limits(job.steps, job.equil)
        job.admitted = now
        return g

    @staticmethod
    def _next_bound(job: Job, step: int) -> int:
        for b in job._bounds:
            if b > step:
                return b
        return job.steps

    @staticmethod
    def _close_blocks(job: Job, g: "native.GpuSystem", step: int):
        """Records the blocks that end at or before `step`, then lets the job
        run to its next block boundary."""
        while len(job._blocks) < len(job._bounds) and job._bounds[len(job._blocks)] <= step:
            cur = output.Block.from_sums(g.averages()["sums"])
            job._blocks.append(cur.minus(job._prev))
            job._prev = cur
        g.set_limits(Server._next_bound(job, step), job.equil)

    @staticmethod
    def _result(job: Job, g: "native.GpuSystem") -> dict:
        st = g.state()
        av = g.averages()
        kT = units.K_B * job.system.temperature
        out = {"loading": av["loading"], "energy_K": av["energy"] / units.K_B,
               "enthalpy_K": av["enthalpy"] / units.K_B if np.isfinite(av["enthalpy"]) else None,
               "samples": av["samples"], "final_nmol": st["nmol"], "steps": int(st["step"]),
               "status": st["status"], "energy_terms": st["energy"][:6].tolist(),
               "counters": st["counters"][:10].tolist(), "kT": kT}
        if job.keep_checkpoint:
            out["checkpoint"] = g.checkpoint()
        if job.raspa_output:
            out["blocks"] = list(job._blocks)
            out["raspa_summary"] = output.summary_text(job.system, job._blocks)
        return out

    def run(self, jobs: Sequence[Job], realtime: bool = True) -> dict:
        """Serves `jobs` (arrival times relative to the call) to completion.
        With realtime=False every job is available at once. Returns the
        latency and throughput figures; per-job results are on the jobs.

        Admission runs on a host thread of its own: it sets up each arrived
        job's system (device allocation, upload, structure factors, on the
        system's own stream) while this thread launches and retires, for
        the free slots plus `lookahead` more. The engine has max_slots slots
        from its first build; the free ones hold an idle placeholder system
        sized for the job list (`_placeholder`), and a finished job's system
        stays in its slot (at its step limit it takes no step). A new job's
        system replaces one of them in place (Engine.replace: no allocation,
        no device synchronisation, the captured graph stays valid). A new
        engine is built only when a system does not fit the engine's layout.
        Replaced systems are freed in batches, when the device is idle
        anyway."""
        import threading

        import torch

        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        slots: List[Optional[list]] = []     # engine slot -> [job, GpuSystem, steps done, footprint] or None
        occupants: List["native.GpuSystem"] = []   # the system in each slot (a finished job's until replaced)
        unplaced: List[list] = []            # admitted, not yet in the engine
        to_free: List["native.GpuSystem"] = []
        eng = None
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        total_steps = 0
        busy = 0.0
        max_active = 0
        rebuilds = 0
        replacements = 0
        host = collections.defaultdict(float)   # host seconds by phase
        holder = self._placeholder(jobs)

        # shared with the admission thread, under `cond`
        cond = threading.Condition()
        adm = {"mem": 0, "busy": 0, "held": 0, "left": len(jobs), "error": None}
        ready: collections.deque = collections.deque()   # set up, handed to this thread
        stop = threading.Event()
        fps = {id(j): footprint_bytes(j) for j in jobs}

        def admission():
            """sets up arrived jobs while slots (plus lookahead) and the
            memory budget allow; busy = jobs in slots, held = admitted
            jobs not yet in a slot (set up or being set up). Waits on `cond`
            for the next arrival or for jobs to finish."""
            try:
                while not stop.is_set() and pending:
                    job = None
                    with cond:
                        fp = fps[id(pending[0])]
                        n = adm["busy"] + adm["held"]
                        arrived = pending[0].arrival <= now() or not realtime
                        if arrived and n < self.max_slots + self.lookahead and \
                                (adm["mem"] + fp <= self.mem_budget or n == 0):
                            job = pending.popleft()
                            adm["mem"] += fp
                            adm["held"] += 1
                        else:
                            wait = pending[0].arrival - now() if not arrived else 0.05
                            cond.wait(timeout=max(wait, 1e-4))
                    if job is None:
                        continue
                    h0 = time.perf_counter()
                    g = self._admit(job, now())
                    entry = [job, g, int(g.state()["step"]) if job.resume is not None else 0, fp]
                    with cond:
                        ready.append(entry)
                        host["admit"] += time.perf_counter() - h0
                        cond.notify_all()
            except BaseException as e:  # surfaced by the serving loop
                with cond:
                    adm["error"] = e

        def place():
            """the admitted jobs into free slots, or a new engine; jobs
            admitted ahead wait while every slot is busy"""
            nonlocal eng, slots, occupants, rebuilds, replacements
            rest, wait_slot = [], []
            for entry in unplaced:
                i = next((k for k, a in enumerate(slots) if a is None), None)
                if eng is not None and i is None:
                    wait_slot.append(entry)
                elif eng is not None and eng.replace(i, entry[1], self.stream.cuda_stream):
                    if occupants[i] is not holder:
                        to_free.append(occupants[i])
                    slots[i], occupants[i] = entry, entry[1]
                    entry[0].started = now()
                    replacements += 1
                else:
                    rest.append(entry)
            free = self.max_slots - sum(1 for a in slots if a is not None)
            unplaced[:] = wait_slot + rest[max(free, 0):]
            rest = rest[:max(free, 0)]
            if rest:
                # a new engine: the active jobs, the new ones, and the finished
                # jobs' systems still held (their slots stay free for later jobs)
                keep = [(a, g) for a, g in zip(slots, occupants)]
                keep = [(a, g) for a, g in keep if a is not None] + [(e, e[1]) for e in rest] + \
                       [(a, g) for a, g in keep if a is None]
                keep = keep[:max(self.max_slots, sum(1 for a, _ in keep if a is not None))]
                held = {id(g) for _, g in keep}
                to_free.extend(g for g in occupants if id(g) not in held and g is not holder)
                if holder is not None:
                    keep += [(None, holder)] * (self.max_slots - len(keep))
                slots = [a for a, _ in keep]
                occupants = [g for _, g in keep]
                for e in rest:
                    e[0].started = now()
                if eng is not None:
                    eng.close()
                eng = native.Engine(occupants, precision=self.precision, threads=self.threads, cluster=self.cluster)
                eng.use_graph(True)
                rebuilds += 1
            n_busy = sum(1 for a in slots if a is not None)
            with cond:
                adm["held"] -= n_busy - adm["busy"]
                adm["busy"] = n_busy
                cond.notify_all()

        # no cyclic garbage collection while serving: a full collection of a
        # large process holds the interpreter lock for tens of milliseconds,
        # and the serving loop would miss its next launch meanwhile
        gc_on = gc.isenabled()
        gc.collect()
        gc.disable()
        worker = threading.Thread(target=admission, name="raspa2-admission", daemon=True)
        worker.start()
        try:
            while True:
                with cond:
                    if adm["error"] is not None:
                        raise adm["error"]
                    while ready:
                        unplaced.append(ready.popleft())
                    left = adm["left"]
                h1 = time.perf_counter()
                if unplaced:
                    place()
                host["place"] += time.perf_counter() - h1
                running = [a for a in slots if a is not None]
                if not running:
                    if left == 0:
                        break
                    with cond:                                # the admission thread is setting jobs up
                        if not ready and adm["error"] is None:
                            cond.wait(timeout=5e-3)
                    continue
                max_active = max(max_active, len(running))
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record(self.stream)
                eng.run(self.chunk, self.stream.cuda_stream)      # asynchronous
                ev1.record(self.stream)
                self.launches += 1
                h1 = time.perf_counter()
                eng.sync()
                ev1.synchronize()
                h2 = time.perf_counter()
                host["wait"] += h2 - h1
                busy += ev0.elapsed_time(ev1) / 1e3               # device time of the launch
                freed_mem, finished = 0, 0
                for k, a in enumerate(slots):
                    if a is None:
                        continue
                    job, g, done, fp = a
                    if job.raspa_output:
                        # the engine stopped the job at its block boundary or ran the chunk
                        step = int(g.state()["step"])
                        adv = step - done
                        self._close_blocks(job, g, step)
                    else:
                        adv = min(self.chunk, job.steps - done)   # the engine stops each job at its limit
                    total_steps += adv
                    a[2] = done + adv
                    if a[2] >= job.steps:
                        job.result = self._result(job, g)
                        job.finished = now()
                        freed_mem += fp
                        finished += 1
                        slots[k] = None                           # the system stays in the slot, idle
                if finished:
                    with cond:
                        adm["mem"] -= freed_mem
                        adm["busy"] -= finished
                        adm["left"] -= finished
                        cond.notify_all()
                h3 = time.perf_counter()
                host["results"] += h3 - h2
                if len(to_free) >= 32:
                    for g in to_free:
                        g.close()
                    to_free.clear()
                host["free"] += time.perf_counter() - h3
        finally:
            stop.set()
            with cond:
                cond.notify_all()
            worker.join()
            if gc_on:
                gc.enable()
        if eng is not None:
            eng.close()
        for g in set(to_free + occupants + list(e[1] for e in unplaced) + ([holder] if holder is not None else [])):
            g.close()
        torch.cuda.synchronize()
        makespan = now()
        lat = np.array([j.latency for j in jobs]) * 1e3
        wait = np.array([j.started - j.arrival for j in jobs]) * 1e3
        span = max(j.arrival for j in jobs) - min(j.arrival for j in jobs) if realtime and len(jobs) > 1 else 0.0
        req = float(sum(j.steps for j in jobs))
        return {"jobs": len(jobs), "makespan_s": makespan, "launches": self.launches,
                "p50_job_ms": float(np.percentile(lat, 50)), "p99_job_ms": float(np.percentile(lat, 99)),
                "p50_wait_ms": float(np.percentile(wait, 50)), "p99_wait_ms": float(np.percentile(wait, 99)),
                "mc_steps": int(total_steps), "mc_steps_per_s": total_steps / makespan, "max_active": max_active,
                "p50_service_ms": float(np.percentile([(j.finished - j.started) * 1e3 for j in jobs], 50)),
                "gpu_busy_frac": busy / makespan,
                "offered_steps_per_s": req / span if span > 0 else None,
                "engine_builds": rebuilds, "slot_replacements": replacements,
                "host_s": {k: round(v, 4) for k, v in host.items()}}


# --------------------------------------------------------------------------
# served workload: Poisson stream of methane / CO2 isotherm points

def _framework_templates(n_each: int, seed: int) -> List[systems.System]:
    """Distinct frameworks the jobs draw from: methane-type (neutral, the
    config-0 density) and CO2-type (charged, the config-1 density), sizes
    log-spaced over 288-4096 atoms."""
    rng = np.random.default_rng(seed)
    out = []
    sizes = np.unique(np.round(np.geomspace(288, 4096, n_each)).astype(int))
    for i, n in enumerate(sizes):
        out.append(systems.methane_like_system(seed=seed * 100 + i, n_atoms=int(n)))
        cell = 25.8 * (n / 1536.0) ** (1.0 / 3.0)
        out.append(systems.co2_system(seed=seed * 100 + 50 + i, n_atoms=int(n), cell=float(cell),
                                      kmax=int(rng.integers(6, 11)), name=f"co2_served{i}"))
    return out


def served_jobs(n: int, rate: float = 200.0, seed: int = 3, cycles=(500, 3000),
                templates: Optional[List[systems.System]] = None) -> List[Job]:
    """`n` jobs arriving as a Poisson stream of `rate` jobs/s. Each job is a
    state point (pressure log-uniform 1e3-1e7 Pa, T in {273, 298, 323} K) of
    one of the framework templates, run for a uniform number of cycles in
    `cycles`; a cycle is 20 MC steps (the reference's minimum per cycle);
    the first third is equilibration."""
    rng = np.random.default_rng(seed)
    templates = templates or _framework_templates(8, seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    jobs = []
    for i in range(n):
        base = templates[int(rng.integers(len(templates)))]
        p = float(10.0 ** rng.uniform(3.0, 7.0))
        T = float((273.0, 298.0, 323.0)[int(rng.integers(3))])
        s = dataclasses.replace(base, pressure=p, temperature=T, name=f"{base.name}_j{i}")
        steps = int(rng.integers(cycles[0], cycles[1] + 1)) * RASPA_MIN_STEPS_PER_CYCLE
        jobs.append(Job(id=i, system=s, steps=steps, equil=steps // 3, seed=1000 + i, arrival=float(t[i])))
    return jobs
