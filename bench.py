"""Benchmark: batched mixed-precision GCMC MC moves/s on one node.

Workload (default): 64 independent CO2 GCMC systems of uneven size advanced
by one persistent launch of the batched engine per step: cubic cells 18-36 A
with 512-4096 framework atoms per cell (2x2x2 replication below 24 A),
charges uniform in [-1.2, 1.2] e made neutral, Ewald alpha 0.265/A with kmax
6-10, pressures log-spaced 1e3-1e7 Pa, T in {273, 298, 323} K, rigid 3-site
CO2 with CBMC insertion/deletion (10 first-bead x 10 orientation trials),
translation and rotation; FP32 pair terms with FP64 S(k), totals and
acceptance. Synthetic frameworks, seeded per system.

One step = `--moves-per-step` MC moves attempted by every system (counted as
the reference counts attempted moves). Timing: CUDA events on the engine's
stream around each step, the L2 cache flushed between steps (outside the
events), warm-up steps first; max over ranks; value = moves of all ranks /
that time. With torchrun each rank runs its own 64 systems (weak scaling, no
collective on the data path).

`--impl reference` times the reference's own CPU implementation
(oracle/_ref/simulate, built from the reference sources) on the same systems
on all host cores.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from raspa2_b200 import ranks, raspa_io, systems, units  # noqa: E402

METRIC = "MC moves/sec, batched mixed-prec vs plain GPU at 1e-6 rel err; p50/p99 job ms"
REF_SIMULATE = os.path.join(ROOT, "oracle", "_ref", "simulate")

# algorithmic FLOP per unit of work (counting FMA = 2, MUFU = 1)
FLOP_PAIR_LJ = 25.0        # in-cutoff pair, LJ only
FLOP_PAIR_LJ_EWALD = 49.0  # in-cutoff pair, LJ + real-space Ewald
FLOP_KSITE = 10.0          # dS(k) per (wave vector, moved site)
FLOP_KVEC = 12.0           # FP64 energy terms per wave vector


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nsys", type=int, default=64)
    p.add_argument("--moves-per-step", type=int, default=2000)
    p.add_argument("--threads", type=int, default=0, help="CTA size; 0 = autotuned")
    p.add_argument("--cluster", type=int, default=0, help="CTAs per system; 0 = autotuned")
    p.add_argument("--maxmol", type=int, default=768)
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "mixed_cc64"])
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--ref-cycles", type=int, default=2,
                   help="reference production cycles per system and step (a cycle is max(20, N) moves)")
    p.add_argument("--single-ref-cycles", type=int, default=20,
                   help="reference production cycles of each single-system configuration")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--hexane-systems", type=int, default=64,
                   help="systems of the grid-accelerated hexane workload (0 = skip)")
    p.add_argument("--hexane-moves", type=int, default=1000, help="moves per system per timed hexane step")
    p.add_argument("--hexane-spacing", type=float, default=0.1, help="energy-grid spacing of the hexane workload [A]")
    p.add_argument("--serve-jobs", type=int, default=300, help="jobs of the served Poisson stream (0 = skip)")
    p.add_argument("--serve-rate", type=float, default=200.0, help="mean arrivals per second")
    p.add_argument("--serve-steady-rate", type=float, default=25.0,
                   help="arrival rate of the second, below-capacity served stream (0 = skip)")
    p.add_argument("--serve-steady-jobs", type=int, default=100)
    return p.parse_args()


# --------------------------------------------------------------------------
# reference CPU implementation
def reference_sample(systems_list, cycles, seed0, workdir, cores):
    """Runs the reference `simulate` on every system (one process each, `cores`
    at a time) for `cycles` production cycles from an empty framework and
    parses the attempted moves and the MC-move CPU seconds of each run."""
    dirs = []
    for i, s in enumerate(systems_list):
        d = os.path.join(workdir, f"s{i}")
        raspa_io.write_inputs(s, d, cycles=cycles, init_cycles=0, print_every=10 ** 9, seed=seed0 + i)
        dirs.append(d)

    def run(d):
        t0 = time.perf_counter()
        r = subprocess.run([REF_SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference simulate failed in {d}: {r.stderr[-500:]}")
        out = os.path.join(d, "Output", "System_0")
        f = os.path.join(out, os.listdir(out)[0])
        return parse_reference_output(f) + (wall,)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as ex:
        res = list(ex.map(run, dirs))
    pool_wall = time.perf_counter() - t0
    moves = sum(r[0] for r in res)
    cpu = sum(r[1] for r in res)
    return moves, cpu, pool_wall, res


def parse_reference_output(path):
    txt = open(path).read()
    moves = 0.0
    for name in ("translation", "rotation"):
        m = re.search(r"Performance of the %s move:\n=+\nComponent 0 \[[^\]]*\]\n\s*total\s+([\d.eE+-]+)\s+([\d.eE+-]+)\s+([\d.eE+-]+)" % name, txt)
        if m:
            moves += sum(float(x) for x in m.groups())
    for name in ("swap addition", "swap deletion"):
        m = re.search(r"Performance of the %s move:\n=+\nComponent \[[^\]]*\] total tried: ([\d.eE+-]+)" % name, txt)
        if m:
            moves += float(m.group(1))
    blk = txt.split("Production run CPU timings of the MC moves:")[1].split("Total all components:")[0]
    cpu = 0.0
    for key in ("translation", "rotation", "swap (insertion)", "swap (deletion)"):
        m = re.search(r"\n\s*%s:\s+([\d.eE+-]+) \[s\]" % re.escape(key), blk)
        if m:
            cpu += float(m.group(1))
    return moves, cpu


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def equilibrated_configs(args, sys_list):
    """The GPU arm's starting state, reproduced: every system from empty
    through the GPU arm's warm-up (warmup + 1 steps of moves_per_step MC
    moves, the same seeds and random streams; a system's trajectory does not
    depend on the launch shape or the batch) on the engine. Returns the
    configurations, or None when no GPU or library is there."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        from raspa2_b200 import native
        native.load()
    except Exception:
        return None
    gs = [native.GpuSystem(s, maxmol=args.maxmol, seed=20240, stream_id=i) for i, s in enumerate(sys_list)]
    for g, s in zip(gs, sys_list):
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
    prec = {"mixed": native.RGPU_MIXED, "fp64": native.RGPU_FP64, "mixed_cc64": native.RGPU_MIXED_CC64}[args.precision]
    eng = native.Engine(gs, precision=prec, threads=512, cluster=0)   # one GPU: stream ids = batch order
    for _ in range(args.warmup + 1):
        eng.run(args.moves_per_step)
    eng.sync()
    xs = [g.adsorbates() for g in gs]
    eng.close()
    return xs


def run_reference_arm(args, sys_list):
    if not os.path.exists(REF_SIMULATE):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/simulate was not built "
                                                              "(needs the reference sources: make -C oracle ref)"}))
        return
    cores = min(cpu_cores(), len(sys_list))
    xs = equilibrated_configs(args, sys_list)
    start = "the GPU arm's equilibrated configuration of each system (restart file)" if xs is not None else \
        "empty framework (no GPU to equilibrate on)"
    if xs is None:
        xs = [np.zeros((0, s.molecule.n_atoms, 3)) for s in sys_list]
    tmp = tempfile.mkdtemp(prefix="raspa_ref_")
    n = len(sys_list)
    try:
        def sample(k, cycles, tag):
            idx = [(k * cores + j) % n for j in range(cores)]
            return idx, reference_from([(sys_list[i], xs[i]) for i in idx], cycles, 1000 + 97 * k,
                                       os.path.join(tmp, f"{tag}{k}"), cores)
        for w in range(args.warmup):
            sample(w, 1, "w")
        total_moves, total_cpu, total_wall, loads, seen = 0.0, 0.0, 0.0, {}, []
        for k in range(args.steps):
            t0 = time.perf_counter()
            idx, res = sample(k, args.ref_cycles, "k")
            total_wall += time.perf_counter() - t0
            for i, (mv, cpu, wall, ld) in zip(idx, res):
                total_moves += mv
                total_cpu += cpu
                loads[i] = ld
                seen.append(i)
        per_core = total_moves / total_cpu
        value = per_core * cores
        sampled = sorted(loads)
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "MC moves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * total_wall / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"co2_gcmc_batched_{n}", "systems_per_gpu": n,
                       "moves_per_step_per_system": f"{args.ref_cycles} cycles of max(20, N) moves",
                       "precision": "fp64", "start": start,
                       "mean_loading": float(np.mean([loads[i] for i in sampled])),
                       "start_mean_loading": float(np.mean([len(xs[i]) for i in sampled])),
                       "systems_sampled": len(sampled)},
            "cpu_baseline": {"value": value, "unit": "MC moves/s", "cores": cores, "kind": "reference",
                             "sample": f"per step {cores} of the {n} systems (in turn), {args.ref_cycles} "
                                       "production cycles each from the equilibrated configuration, one "
                                       "process per system; moves / production MC-move CPU time x cores",
                             "single_core": per_core, "wall_clock_aggregate": total_moves / total_wall},
            "e2e": {"value": value, "unit": "MC moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                s, m, util = float(p[0]), float(p[1]), float(p[6])
            except ValueError:
                continue
            mx = m
            if util > 0:
                sm.append(s)
            for n, v in zip(names, p[2:6]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(self.lines)}


def make_systems(n, rank):
    return systems.batched_co2_systems(n, seed=ranks.batch_seed(2, rank))


def placed_systems(args, world, rank):
    """This rank's systems: the job set of `world` GPUs is the union of
    `world` seeded batches of `nsys` systems, placed on the GPUs by
    device-memory footprint (ranks.place, the same on every rank), at most
    nsys per GPU. Returns (systems, their indices in the job set); with one
    GPU, the one batch in order."""
    from raspa2_b200 import serve
    allsys = [s for r in range(world) for s in make_systems(args.nsys, r)]
    fp = [serve.system_footprint_bytes(s, args.maxmol) for s in allsys]
    work = [float(s.n_framework() + (len(systems.kvector_indices(s.kmax)) if s.ewald else 0)) for s in allsys]
    mine = ranks.place(fp, work, world, max_items=args.nsys)[rank]
    return [allsys[i] for i in mine], mine


def energy_error(gs, sys_list):
    """The engine's running energies (accumulated move by move) of every
    system against an FP64 recomputation of its configuration from scratch
    (rgpu_total_energy; rgpu_intra_energy for chains): the largest plain
    relative error of the total potential energy and of each term larger
    than k_B T, and the largest absolute differences in k_B T."""
    rel_tot, abs_tot, rel_term, abs_term, per_mol, n = 0.0, 0.0, 0.0, 0.0, 0.0, 0
    for g, s in zip(gs, sys_list):
        st = g.state()
        if st["nmol"] == 0:
            continue
        n += 1
        run = np.array(st["energy"][:6])
        ref = np.array(g.total_energy())
        if not s.molecule.rigid:
            run = np.append(run, st["energy"][6])
            ref = np.append(ref, g.intra_energy())
        kT = units.K_B * s.temperature
        d = abs(run.sum() - ref.sum())
        rel_tot = max(rel_tot, d / abs(ref.sum()))
        abs_tot = max(abs_tot, d / kT)
        per_mol = max(per_mol, d / kT / st["nmol"])
        for a, b in zip(run, ref):
            if abs(b) > kT:
                rel_term = max(rel_term, abs(a - b) / abs(b))
                abs_term = max(abs_term, abs(a - b) / kT)
    return {"systems": n, "max_rel_total": rel_tot, "max_abs_total_kT": abs_tot,
            "max_abs_total_kT_per_molecule": per_mol, "max_rel_term": rel_term, "max_abs_term_kT": abs_term,
            "reference": "FP64 recomputation from scratch of each system's final configuration"}


def roofline_of(d, seconds, peak):
    """FP32 roofline of an engine run from its counter deltas d (summed over
    systems) and its device time."""
    n_charged = float(d[12])
    n_lj = float(d[11]) - n_charged
    flop = FLOP_PAIR_LJ * n_lj + FLOP_PAIR_LJ_EWALD * n_charged + FLOP_KSITE * float(d[13]) + FLOP_KVEC * float(d[14])
    achieved = flop / seconds / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak}


def write_restart_inputs(s, d, xyz, cycles, seed):
    """Input files of system s in directory d for a production run of the
    reference that starts from the configuration xyz ([n][natom][3]) through
    its restart file (RestartFile yes)."""
    from raspa2_b200 import restart
    raspa_io.write_inputs(s, d, cycles=cycles, init_cycles=0, print_every=1, seed=seed, restart=True)
    restart.write_restart(restart.restart_path(s, d), s, np.asarray(xyz, float).reshape(-1, s.molecule.n_atoms, 3))
    return d


def reference_from(sys_xyz, cycles, seed0, workdir, cores):
    """The reference `simulate` on each (system, configuration), one process
    per system, `cores` at a time, each for `cycles` production cycles from
    its configuration; returns per run (moves, MC-move CPU s, wall s, mean
    loading in molecules per box)."""
    dirs = []
    for i, (s, x) in enumerate(sys_xyz):
        dirs.append((s, write_restart_inputs(s, os.path.join(workdir, f"s{i}"), x, cycles, seed0 + i)))

    def run(sd):
        s, d = sd
        t0 = time.perf_counter()
        r = subprocess.run([REF_SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference simulate failed in {d}: {r.stderr[-500:]}")
        out = os.path.join(d, "Output", "System_0")
        f = os.path.join(out, os.listdir(out)[0])
        mv, cpu = parse_reference_output(f)
        # the running average of the molecule count the reference prints
        # every cycle (its block averages need five blocks of cycles)
        m = re.findall(r"current number of integer/fractional/reaction molecules: \d+/\d+/\d+ \(avg\.\s+([-\d.eE+]+)\)",
                       open(f).read())
        return mv, cpu, wall, float(m[-1]) if m else float("nan")

    with ThreadPoolExecutor(max_workers=cores) as ex:
        return list(ex.map(run, dirs))


def run_ours(args):
    import torch
    import torch.distributed as dist
    from raspa2_b200 import native

    world, rank, local = ranks.rank_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    prec = {"mixed": native.RGPU_MIXED, "fp64": native.RGPU_FP64, "mixed_cc64": native.RGPU_MIXED_CC64}[args.precision]

    sys_list, sys_ids = placed_systems(args, world, rank)
    gs = [native.GpuSystem(s, maxmol=args.maxmol, seed=20240, stream_id=i) for i, s in zip(sys_ids, sys_list)]
    for g, s in zip(gs, sys_list):
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
    eng = native.Engine(gs, precision=prec, threads=args.threads or 512, cluster=args.cluster)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    def counters():
        return np.array([g.state()["counters"] for g in gs])

    # warm-up (equilibrates the loadings)
    for _ in range(args.warmup):
        eng.run(args.moves_per_step, stream.cuda_stream)
    torch.cuda.synchronize()
    # launch shape: autotuned on copies of the equilibrated systems unless
    # both are given; the engine is rebuilt with the chosen shape and warmed
    shape = {"cluster": eng.cluster, "threads": eng.threads, "tuned": False}
    if not (args.threads and args.cluster):
        from raspa2_b200 import autotune
        tuned = autotune.tune(gs, precision=prec)
        shape = dict(tuned.describe(), tuned=True, table=tuned.table)
        eng.close()
        eng = tuned.engine(gs, prec)
        eng.run(args.moves_per_step, stream.cuda_stream)
        torch.cuda.synchronize()
    c0 = counters()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        t_wall0 = time.perf_counter()
        torch.cuda.nvtx.range_push("timed")       # the launch list of a profiler filters on this range
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                evs[k][0].record(stream)
                eng.run(args.moves_per_step, stream.cuda_stream)
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        t_wall = time.perf_counter() - t_wall0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    t_dev = sum(ms) / 1000.0
    c1 = counters()
    d = (c1 - c0).sum(axis=0)
    moves = float(d[8])
    status = [g.state()["status"] for g in gs]
    t_dev_max, moves_all = ranks.reduce_time_and_count(t_dev, moves, dev)
    value = moves_all / t_dev_max

    # roofline of the engine kernel (one launch per step)
    n_charged = float(d[12])
    n_lj = float(d[11]) - n_charged
    flop = FLOP_PAIR_LJ * n_lj + FLOP_PAIR_LJ_EWALD * n_charged + FLOP_KSITE * float(d[13]) + FLOP_KVEC * float(d[14])
    achieved = flop / t_dev / 1e12
    peak = native.fp32_peak_tflops()

    # end to end through the public API with host buffers: every step uploads
    # every system's configuration from host memory, runs, and reads back
    # every system's state block and positions, one batched transfer each way
    e2e = None
    if args.e2e_steps > 0:
        torch.cuda.synchronize()
        states = eng.get_states()
        xs = [st["xyz"].copy() for st in states]
        prev = sum(int(st["counters"][8]) for st in states)
        stage = eng.staging_bytes()
        moves_e = 0.0
        t0 = time.perf_counter()
        torch.cuda.nvtx.range_push("e2e")
        for _ in range(args.e2e_steps):
            eng.set_adsorbates(xs)
            eng.run(args.moves_per_step, stream.cuda_stream)
            states = eng.get_states()
            xs = [st["xyz"] for st in states]
            tot = sum(int(st["counters"][8]) for st in states)
            moves_e += tot - prev
            prev = tot
        torch.cuda.nvtx.range_pop()
        t_e = time.perf_counter() - t0
        t_e, moves_e = ranks.reduce_time_and_count(t_e, moves_e, dev)
        e2e = {"value": moves_e / t_e, "unit": "MC moves/s",
               "h2d_bytes_per_step": int(stage), "d2h_bytes_per_step": int(stage),
               "path": "rgpu_engine_set_adsorbates + rgpu_engine_run + rgpu_engine_get_state per step "
                       "(host configurations in, every state block and position out)"}

    loads = [g.state()["nmol"] for g in gs]
    cyc = (c1 - c0)[:, 15].astype(float)
    imbalance = {"max_over_mean_system_cycles": float(cyc.max() / max(cyc.mean(), 1.0)),
                 "slowest_system": int(np.argmax(cyc)), "slowest_atoms": int(sys_list[int(np.argmax(cyc))].n_framework()),
                 "slowest_loading": int(loads[int(np.argmax(cyc))]),
                 "us_per_move_mean": float(np.mean(cyc / np.maximum((c1 - c0)[:, 8], 1)) / 1965.0),
                 "share_eval": float((c1 - c0)[:, 16].sum() / max(cyc.sum(), 1.0)),
                 "share_ewald": float((c1 - c0)[:, 17].sum() / max(cyc.sum(), 1.0))}
    line = {
        "metric": METRIC, "value": value, "unit": "MC moves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": {native.RGPU_MIXED: "f32", native.RGPU_FP64: "f64"}.get(prec, "f32+f64"),
        "data": "synthetic (seeded frameworks, random-init adsorbate state)",
        "config": {"workload": f"co2_gcmc_batched_{args.nsys}", "systems_per_gpu": args.nsys,
                   "placement": "job set of n_gpus seeded batches, placed by device-memory footprint "
                                "(ranks.place), no collective on the data path",
                   "moves_per_step_per_system": args.moves_per_step, "launch_shape": shape,
                   "precision": args.precision, "l2": "flushed between timed steps (256 MB write)",
                   "framework_atoms": [int(s.n_framework()) for s in sys_list[:8]] + ["..."],
                   "mean_loading": float(np.mean(loads))},
        "wall_s": t_wall, "gpu_launches": args.steps * (2 if eng.split[0] else 1),
        "status_nonzero_systems": int(sum(1 for s in status if s)),
        "load_balance": imbalance, "cluster": eng.cluster,
        "acceptance": {k: (float(d[4 + i]) / max(float(d[i]), 1.0)) for i, k in
                       enumerate(["translation", "rotation", "insertion", "deletion"])},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": "measured FP32 FMA probe (rgpu_fp32_peak_probe) on this GPU",
                     "work": {"pairs_in_cutoff_lj": n_lj, "pairs_in_cutoff_lj_ewald": n_charged,
                              "pairs_visited": float(d[10]), "k_site_products": float(d[13]),
                              "k_energy_terms": float(d[14])}},
        "clocks": clk.summary(),
    }
    if e2e:
        line["e2e"] = e2e
    line["precision"] = {"co2_batched": energy_error(gs, sys_list)}
    if rank == 0 and world == 1 and not args.no_plain and prec == native.RGPU_MIXED:
        line["batched_fp64"] = batched_fp64_run(native, stream, gs, sys_list, args, peak)
        # the mixed engine and its variant with FP64 real-space charge-charge
        # terms over the same number of moves from the same anchored start:
        # their moves/s and the error their running energies accumulate
        for key, p in (("batched_mixed_cc64", native.RGPU_MIXED_CC64), ("batched_mixed_anchored", native.RGPU_MIXED)):
            line[key] = batched_fp64_run(native, stream, gs, sys_list, args, peak, steps=args.steps, precision=p)
        line["precision"]["co2_batched_cc64"] = line["batched_mixed_cc64"]["energy_error"]
        line["precision"]["co2_batched_mixed_anchored"] = line["batched_mixed_anchored"]["energy_error"]
        # the metric's error bound, engine by engine: moves/s and the largest
        # relative error of a box's running total energy
        line["at_1e-6_rel_err"] = {
            k: {"moves_per_s": float(v), "max_rel_total": float(e), "within": bool(e <= 1e-6)} for k, v, e in (
                ("mixed", value, line["precision"]["co2_batched"]["max_rel_total"]),
                ("mixed_cc64", line["batched_mixed_cc64"]["moves_per_s"],
                 line["precision"]["co2_batched_cc64"]["max_rel_total"]),
                ("fp64", line["batched_fp64"]["moves_per_s"], line["batched_fp64"]["energy_error"]["max_rel_total"]))}
    if rank == 0 and world == 1 and not args.no_plain:
        line["plain_gpu"] = plain_gpu_rate(native, stream)
        # the two single-system configurations, each on its own
        line["config0_methane"] = single_config_run(native, stream, peak, systems.methane_system(seed=0), 256,
                                                    60000, 20000, args.single_ref_cycles)
        line["config1_co2"] = single_config_run(native, stream, peak, systems.co2_system(seed=1), 384, 200000,
                                                20000, args.single_ref_cycles)
        line["precision"]["config0_methane"] = line["config0_methane"]["mixed"]["energy_error"]
        line["precision"]["config1_co2"] = line["config1_co2"]["mixed"]["energy_error"]
    if rank == 0 and world == 1 and args.serve_jobs > 0:
        line["serving"] = serving_run(args)
    if rank == 0 and world == 1 and args.hexane_systems > 0:
        line["hexane_grid"] = hexane_grid_run(args, stream)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_SIMULATE):
        # the reference on the GPU arm's final configurations: the first
        # `cores` systems, one process each, 2 production cycles
        cores = min(cpu_cores(), len(sys_list))
        tmp = tempfile.mkdtemp(prefix="raspa_ref_")
        try:
            res = reference_from([(sys_list[i], gs[i].adsorbates()) for i in range(cores)], args.ref_cycles, 4242,
                                 tmp, cores)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        per_core = sum(r[0] for r in res) / sum(r[1] for r in res)
        line["cpu_baseline"] = {"value": per_core * cores, "unit": "MC moves/s", "cores": cores,
                                "kind": "reference",
                                "sample": f"{cores} of the {len(sys_list)} systems x {args.ref_cycles} production "
                                          "cycles from this run's final configurations, reference simulate "
                                          "(oracle/_ref), one process per system",
                                "single_core": per_core,
                                "mean_loading": float(np.mean([r[3] for r in res])),
                                "gpu_mean_loading_same_systems": float(np.mean(loads[:cores]))}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def serving_run(args):
    """The served workload: a Poisson stream of methane / CO2 isotherm-point
    jobs (frameworks of 288-4096 atoms per unit cell, 500-3000 cycles of 20
    MC steps, pressures 1e3-1e7 Pa) through the continuous-batching server.
    Latency = finish - arrival, wall clock, including queueing."""
    from raspa2_b200 import serve
    jobs = serve.served_jobs(args.serve_jobs, rate=args.serve_rate, seed=3)
    srv = serve.Server()
    st = srv.run(jobs, realtime=True)
    st.update({"workload": "served isotherm points (methane/CO2)", "arrival_rate_jobs_per_s": args.serve_rate,
               "launch_shape": {"cluster": srv.cluster, "threads": srv.threads}, "chunk_steps": srv.chunk,
               "slots": srv.max_slots, "mem_budget_gb": srv.mem_budget / 1e9,
               "status_nonzero_jobs": int(sum(1 for j in jobs if j.result["status"]))})
    # the same stream at an offered load below what the server serves: the
    # latencies of a steady state rather than of a queue behind a burst
    if args.serve_steady_rate > 0:
        jobs2 = serve.served_jobs(args.serve_steady_jobs, rate=args.serve_steady_rate, seed=5)
        st2 = serve.Server().run(jobs2, realtime=True)
        st2.update({"arrival_rate_jobs_per_s": args.serve_steady_rate,
                    "status_nonzero_jobs": int(sum(1 for j in jobs2 if j.result["status"]))})
        st["steady_state"] = st2
    return st


def hexane_grid_run(args, stream, steps=3, warmup=3):
    """Grid-accelerated CBMC of united-atom n-hexane: one 4096-atom neutral
    framework in a cubic 40 A cell at 64 pressures (1e2-1e6 Pa, T = 433 K),
    one system per pressure, all sharing the two bead-type energy grids
    (0.1 A: 401^3 points x 8 FP32 values = 2.06 GB each), mixed precision,
    8 first-bead x 16 trials. Device-timed moves/s, then the running host VDW
    energy of every system against direct FP64 pair sums of its final
    configuration."""
    import torch
    from raspa2_b200 import native
    base = systems.hexane_system(seed=4, n_atoms=4096, cell=40.0, temperature=433.0)
    pressures = np.logspace(2, 6, args.hexane_systems)
    sl = [dataclasses.replace(base, pressure=float(p)) for p in pressures]
    gs = [native.GpuSystem(s, maxmol=256, seed=9000, stream_id=i) for i, s in enumerate(sl)]
    t0 = time.perf_counter()
    geom = gs[0].use_energy_grids(args.hexane_spacing)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    for g in gs[1:]:
        g.use_energy_grids(args.hexane_spacing, like=gs[0])
    for g in gs:
        g.set_adsorbates(np.zeros((0, 6, 3)))
    from raspa2_b200 import autotune
    e = native.Engine(gs, precision=native.RGPU_MIXED, threads=512, cluster=1)
    for _ in range(warmup):
        e.run(args.hexane_moves, stream.cuda_stream)
    e.sync()
    tuned = autotune.tune(gs, precision=native.RGPU_MIXED)
    e.close()
    e = tuned.engine(gs, native.RGPU_MIXED)
    e.run(args.hexane_moves, stream.cuda_stream)
    e.sync()
    c0 = np.array([g.state()["counters"] for g in gs])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=stream.device)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.nvtx.range_push("hexane_timed")
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            evs[k][0].record(stream)
            e.run(args.hexane_moves, stream.cuda_stream)
            evs[k][1].record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    t = sum(a.elapsed_time(b) for a, b in evs) / 1e3
    dc = np.array([g.state()["counters"] for g in gs]) - c0
    d = dc.sum(axis=0)
    moves = float(d[8])
    cyc = dc[:, 15].astype(float)
    phases = {"us_per_move_mean": float(np.mean(cyc / np.maximum(dc[:, 8], 1)) / 1965.0),
              "share_eval": float(dc[:, 16].sum() / max(cyc.sum(), 1.0))}
    # bead positions looked up per move type: translation/rotation 6 new + 6
    # old, insertion/deletion 8 first-bead + 5 x 16 trials, reinsertion both
    lookups = 12.0 * (d[0] + d[1]) + 88.0 * (d[2] + d[3]) + 176.0 * d[18]
    # direct FP64 pair sums of every final configuration against the running
    # host VDW energy (grids switched off for the recomputation)
    kT = 433.0 * units.K_B
    errs, rel = [], []
    for g in gs:
        st = g.state()
        g.set_grids(None, None, None, None, None)
        direct = g.total_energy()[0]
        g.use_energy_grids(args.hexane_spacing, like=gs[0])
        if st["nmol"] == 0:
            continue
        errs.append(abs(st["energy"][0] - direct) / st["nmol"] / kT)
        rel.append(abs(st["energy"][0] - direct) / abs(direct))
    loads = [g.state()["nmol"] for g in gs]
    e.close()
    out = {"workload": "hexane_grid_cbmc_64 (4096-atom 40 A framework, 64 pressures 1e2-1e6 Pa, 433 K)",
           "systems": len(gs), "moves_per_step_per_system": args.hexane_moves, "steps": steps,
           "moves_per_s": moves / t, "ms_per_step": 1000.0 * t / steps,
           "launch_shape": tuned.describe(),
           "grid": {"spacing_A": args.hexane_spacing, "points_per_axis": [int(x) + 1 for x in geom[0]],
                    "bytes_per_grid": int(np.prod(geom[0].astype(np.int64) + 1) * 32), "types": 2,
                    "build_s": t_build},
           "grid_lookups_per_s_est": lookups / t,
           "grid_bytes_per_s_est": 256.0 * lookups / t,
           "loading_molecules": {"min": int(min(loads)), "max": int(max(loads)), "mean": float(np.mean(loads))},
           "host_vdw_vs_direct_fp64": {"systems_compared": len(errs), "max_abs_per_molecule_kT": float(max(errs)),
                                       "median_rel": float(np.median(rel)), "max_rel": float(max(rel))},
           "acceptance": {k: (float(d[4 + i]) / max(float(d[i]), 1.0)) for i, k in
                          enumerate(["translation", "rotation", "insertion", "deletion"])},
           "reinsertion_acceptance": float(d[19]) / max(float(d[18]), 1.0), "phases": phases}
    del flush
    return out


def batched_fp64_run(native, stream, gs, sys_list, args, peak, steps=3, precision=None):
    """The same batch of systems on the FP64 engine (the plain path's
    arithmetic: FP64 pair terms, erfc and S(k)), or on the engine of
    `precision`, from the mixed run's final configurations with every
    running energy set to an FP64 recomputation, at its own autotuned launch
    shape: device-timed moves/s and the error of its running energies
    against the FP64 recomputation after the `steps` timed steps."""
    import torch
    from raspa2_b200 import autotune
    precision = native.RGPU_FP64 if precision is None else precision
    g64 = [native.GpuSystem(s, maxmol=args.maxmol, seed=777, stream_id=i) for i, s in enumerate(sys_list)]
    for g, src in zip(g64, gs):
        g.set_adsorbates(src.adsorbates())
        g.set_energy(list(g.total_energy()) + [0.0, 0.0])
    tuned = autotune.tune(g64, precision=precision, moves=300, warm=50)
    e = tuned.engine(g64, precision)
    c0 = np.array([g.state()["counters"] for g in g64])
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        evs[k][0].record(stream)
        e.run(args.moves_per_step, stream.cuda_stream)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    t = sum(a.elapsed_time(b) for a, b in evs) / 1e3
    d = (np.array([g.state()["counters"] for g in g64]) - c0).sum(axis=0)
    out = {"moves_per_s": float(d[8]) / t, "launch_shape": tuned.describe(), "steps": steps,
           "moves_per_step_per_system": args.moves_per_step, "roofline_fp32_equivalent": roofline_of(d, t, peak),
           "energy_error": energy_error(g64, sys_list)}
    e.close()
    for g in g64:
        g.close()
    return out


def single_config_run(native, stream, peak, sysm, maxmol, equil, timed, ref_cycles):
    """One system of a single-system configuration (the plain path): the
    system is equilibrated once by the FP64 engine; from that configuration
    the FP64 and the mixed-precision engine each run `timed` MC moves at
    their own autotuned launch shape (device-timed), with the FP32 roofline
    of the run and the error of the running energies against an FP64
    recomputation; and the reference program runs `ref_cycles` production
    cycles from the same configuration on one host core."""
    import torch
    from raspa2_b200 import autotune
    natom = sysm.molecule.n_atoms
    g = native.GpuSystem(sysm, maxmol=maxmol, seed=5, stream_id=0)
    g.set_adsorbates(np.zeros((0, natom, 3)))
    e = native.Engine([g], precision=native.RGPU_FP64, threads=256, cluster=4)
    e.run(equil, stream.cuda_stream)
    e.sync()
    e.close()
    x_eq = g.adsorbates()
    out = {"system": sysm.name, "framework_atoms": int(sysm.n_framework()), "loading": int(len(x_eq)),
           "equilibration_moves": equil, "timed_moves": timed}
    for prec, key in ((native.RGPU_FP64, "fp64"), (native.RGPU_MIXED, "mixed")):
        g = native.GpuSystem(sysm, maxmol=maxmol, seed=6, stream_id=0)
        g.set_adsorbates(x_eq)
        tuned = autotune.tune([g], precision=prec, moves=200, warm=50, split=False)
        g.set_adsorbates(x_eq)
        g.set_energy(list(g.total_energy()) + [g.intra_energy() if not sysm.molecule.rigid else 0.0, 0.0])
        e = tuned.engine([g], prec)
        c0 = g.state()["counters"].copy()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        e.run(timed, stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        t = ev0.elapsed_time(ev1) / 1e3
        d = g.state()["counters"] - c0
        e.close()
        out[key] = {"moves_per_s": float(d[8]) / t, "launch_shape": tuned.describe(),
                    "roofline": roofline_of(d, t, peak), "energy_error": energy_error([g], [sysm])}
    out["mixed_vs_fp64"] = out["mixed"]["moves_per_s"] / out["fp64"]["moves_per_s"]
    if os.path.exists(REF_SIMULATE):
        tmp = tempfile.mkdtemp(prefix="raspa_ref1_")
        try:
            mv, cpu, wall, ld = reference_from([(sysm, x_eq)], ref_cycles, 31, tmp, 1)[0]
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        out["reference_single_core"] = {"moves_per_s": mv / cpu, "moves": mv, "cycles": ref_cycles, "wall_s": wall,
                                        "mean_loading": ld,
                                        "start": "the same equilibrated configuration (restart file)"}
        out["mixed_vs_reference_single_core"] = out["mixed"]["moves_per_s"] / out["reference_single_core"]["moves_per_s"]
    return out


def plain_gpu_rate(native, stream, nsteps=2000):
    """The plain comparator: one system (the 1536-atom CO2 system) at a time,
    FP64, through the same engine at its own best launch shape (autotuned
    for the single system after equilibration). Device-timed."""
    import torch
    from raspa2_b200 import autotune
    s = systems.co2_system(seed=1)
    g = native.GpuSystem(s, maxmol=256, seed=5, stream_id=0)
    g.set_adsorbates(np.zeros((0, 3, 3)))
    e = native.Engine([g], precision=native.RGPU_FP64, threads=256)
    e.run(nsteps, stream.cuda_stream)
    e.sync()
    tuned = autotune.tune([g], precision=native.RGPU_FP64, moves=200, warm=50)
    e.close()
    e = native.Engine([g], precision=native.RGPU_FP64, threads=tuned.threads, cluster=tuned.cluster)
    e.run(200, stream.cuda_stream)
    e.sync()
    c0 = g.state()["counters"][8]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    e.run(nsteps, stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    t = ev0.elapsed_time(ev1) / 1e3
    return {"engine_fp64_single_system_moves_per_s": (g.state()["counters"][8] - c0) / t,
            "launch_shape": {"cluster": tuned.cluster, "threads": tuned.threads},
            "system": "co2 1536 atoms, kmax 8", "loading": int(g.state()["nmol"])}


def main():
    args = parse_args()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        run_reference_arm(args, make_systems(args.nsys, 0))
        return
    run_ours(args)


if __name__ == "__main__":
    main()
