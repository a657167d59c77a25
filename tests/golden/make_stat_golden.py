"""Generates tests/golden/stat_*.json: ensemble averages of whole GCMC runs of
the reference program, the statistical pin of the engine.

Runs in the build container only (it needs oracle/_ref/simulate, built from
the reference's sources by `make -C oracle ref`). Each case runs the
reference on one of the synthetic systems from an empty framework with
`seeds` independent random seeds (one process per seed), then parses each
run's output:

- average absolute loading [molecules/unit cell] and its block error;
- enthalpy of adsorption [K] and its block error.

The JSON keeps every seed's values and their mean and standard error across
seeds. tests/test_gpu_stats.py compares the engine's averages against it.

Henry cases (HENRY_CASES) run Widom test insertions only: into the framework
(average Rosenbluth weight <W>) and into an empty box (the ideal-gas weight
W_IG), each with `seeds` seeds, and store the Henry ratio <W> / W_IG, the
quantity that is independent of how a code draws the bonded part of its CBMC
trials.

    python tests/golden/make_stat_golden.py [--workdir DIR] [case ...]
"""
from __future__ import annotations

import dataclasses
import json
import os
import re
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from raspa2_b200 import raspa_io, systems  # noqa: E402

SIMULATE = os.path.join(ROOT, "oracle", "_ref", "simulate")
OUT = os.path.dirname(os.path.abspath(__file__))

# name -> (builder, state point, initialisation cycles, production cycles)
CASES = {
    "methane_config0_1e5": (lambda: systems.methane_system(seed=0), dict(pressure=1e5, temperature=300.0), 1000, 8000),
    "methane_config0_1e7": (lambda: systems.methane_system(seed=0), dict(pressure=1e7, temperature=300.0), 1000, 3000),
    "co2_config1_1e5": (lambda: systems.co2_system(seed=1), dict(pressure=1e5, temperature=298.0), 4000, 4000),
    # flexible chains: the reference runs with its own ideal-gas Rosenbluth
    # weight, measured first by Widom insertions into an empty box
    "hexane_small_3e4": (lambda: systems.hexane_system(seed=4, n_atoms=1200, cell=26.0),
                         dict(pressure=3e4, temperature=433.0), 2000, 6000),
    "hexane_small_3e3": (lambda: systems.hexane_system(seed=4, n_atoms=1200, cell=26.0),
                         dict(pressure=3e3, temperature=433.0), 2000, 6000),
}
# cases that take the ideal-gas Rosenbluth weight from the Henry fixture of
# the same molecule and temperature (the mean of its empty-box Widom runs)
# instead of measuring it again; run the Henry case first
REUSE_IDEAL = {"hexane_small_3e4": "hexane_small_henry", "hexane_small_3e3": "hexane_small_henry"}
WIDOM_CYCLES = 20000
SEEDS = 8
IDEAL = {}

# name -> (builder, temperature, Widom cycles in the framework, in the empty box)
HENRY_CASES = {
    "hexane_small_henry": (lambda: systems.hexane_system(seed=4, n_atoms=1200, cell=26.0), 433.0, 4000, 4000),
}


def parse(path):
    txt = open(path).read()
    m = re.search(r"Average loading absolute \[molecules/unit cell\]\s+([-\d.eE+]+) \+/-\s+([-\d.eE+]+)", txt)
    loading, loading_err = float(m.group(1)), float(m.group(2))
    blk = txt.split("Enthalpy of adsorption:")[1]
    m = re.search(r"Average\s+([-\d.eE+]+) \+/-\s+([-\d.eE+]+) \[K\]", blk)
    h, h_err = float(m.group(1)), float(m.group(2))
    return {"loading": loading, "loading_err": loading_err, "enthalpy_K": h, "enthalpy_err_K": h_err}


def reference_ideal_gas_rosenbluth(molecule, temperature, workdir):
    """Average Widom Rosenbluth weight of the reference program for the
    molecule alone in an empty box (its IdealGasRosenbluthWeight)."""
    s = systems.empty_box_system(molecule, temperature)
    d = os.path.join(workdir, f"widom_{molecule.name}_{temperature:g}")
    raspa_io.write_inputs(s, d, cycles=WIDOM_CYCLES, init_cycles=0, print_every=10 ** 9, seed=4242)
    r = subprocess.run([SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"simulate failed in {d}: {r.stderr[-500:]}")
    out = os.path.join(d, "Output", "System_0")
    txt = open(os.path.join(out, os.listdir(out)[0])).read()
    m = re.search(r"Average Widom Rosenbluth-weight:\s+([-\d.eE+]+) \+/-\s+([-\d.eE+]+)", txt)
    return float(m.group(1)), float(m.group(2))


def _widom_run(s, d, cycles, seed):
    raspa_io.write_inputs(s, d, cycles=cycles, init_cycles=0, print_every=10 ** 9, seed=seed)
    r = subprocess.run([SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"simulate failed in {d}: {r.stderr[-500:]}")
    out = os.path.join(d, "Output", "System_0")
    txt = open(os.path.join(out, os.listdir(out)[0])).read()
    m = re.search(r"Average Widom Rosenbluth-weight:\s+([-\d.eE+]+) \+/-\s+([-\d.eE+]+)", txt)
    return float(m.group(1))


def run_henry_case(name, workdir):
    build, T, cyc_fw, cyc_ig = HENRY_CASES[name]
    widom = systems.MoveMix(translation=0.0, rotation=0.0, swap_insert=0.0, swap_delete=0.0, widom=1.0)
    fw = dataclasses.replace(build(), temperature=T, moves=widom)
    ig = systems.empty_box_system(fw.molecule, T)
    jobs = [(fw, os.path.join(workdir, f"{name}_fw_{k}"), cyc_fw, 7001 + 13 * k) for k in range(SEEDS)]
    jobs += [(ig, os.path.join(workdir, f"{name}_ig_{k}"), cyc_ig, 8001 + 13 * k) for k in range(SEEDS)]
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        w = list(ex.map(lambda j: _widom_run(*j), jobs))
    wf, wi = np.array(w[:SEEDS]), np.array(w[SEEDS:])
    mf, sf = wf.mean(), wf.std(ddof=1) / np.sqrt(SEEDS)
    mi, si = wi.mean(), wi.std(ddof=1) / np.sqrt(SEEDS)
    doc = {"case": name, "system": fw.name, "temperature_K": T, "seeds": SEEDS,
           "widom_cycles_framework": cyc_fw, "widom_cycles_empty_box": cyc_ig,
           "widom_weight_runs": wf.tolist(), "ideal_gas_runs": wi.tolist(),
           "widom_weight_mean": float(mf), "widom_weight_se": float(sf),
           "ideal_gas_rosenbluth_mean": float(mi), "ideal_gas_rosenbluth_se": float(si),
           "henry_ratio": float(mf / mi), "henry_ratio_se": float(mf / mi * np.hypot(sf / mf, si / mi)),
           "source": "reference simulate (oracle/_ref) built from the reference sources; Widom moves only"}
    with open(os.path.join(OUT, f"stat_{name}.json"), "w") as fh:
        json.dump(doc, fh, indent=1)
    print(name, doc["henry_ratio"], "+-", doc["henry_ratio_se"])


def run_case(name, workdir):
    build, state, init, prod = CASES[name]
    s = dataclasses.replace(build(), **state)
    if not s.molecule.rigid:
        src = os.path.join(OUT, f"stat_{REUSE_IDEAL.get(name, '')}.json")
        if name in REUSE_IDEAL and os.path.exists(src):
            doc = json.load(open(src))
            w, w_err = doc["ideal_gas_rosenbluth_mean"], doc["ideal_gas_rosenbluth_se"]
        else:
            w, w_err = reference_ideal_gas_rosenbluth(s.molecule, s.temperature, workdir)
        s = dataclasses.replace(s, ideal_gas_rosenbluth=w)
        IDEAL[name] = (w, w_err)
    dirs = []
    for k in range(SEEDS):
        d = os.path.join(workdir, f"{name}_{k}")
        raspa_io.write_inputs(s, d, cycles=prod, init_cycles=init, print_every=10 ** 9, seed=9001 + 17 * k)
        dirs.append(d)

    def one(d):
        r = subprocess.run([SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"simulate failed in {d}: {r.stderr[-500:]}")
        out = os.path.join(d, "Output", "System_0")
        return parse(os.path.join(out, os.listdir(out)[0]))

    return s, dirs, one


def main(argv):
    work = None
    if argv[:1] == ["--workdir"]:
        work, argv = argv[1], argv[2:]
        os.makedirs(work, exist_ok=True)
    names = argv or list(CASES) + list(HENRY_CASES)
    work = work or tempfile.mkdtemp(prefix="raspa_stat_")
    for name in [n for n in names if n in HENRY_CASES]:
        run_henry_case(name, work)
    names = [n for n in names if n not in HENRY_CASES]
    jobs = []
    meta = {}
    for name in names:
        s, dirs, one = run_case(name, work)
        meta[name] = s
        jobs += [(name, d, one) for d in dirs]
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        res = list(ex.map(lambda j: (j[0], j[2](j[1])), jobs))
    for name in names:
        s = meta[name]
        build, state, init, prod = CASES[name]
        runs = [r for n, r in res if n == name]
        L = np.array([r["loading"] for r in runs])
        H = np.array([r["enthalpy_K"] for r in runs])
        doc = {
            "case": name, "system": s.name, "pressure_Pa": s.pressure, "temperature_K": s.temperature,
            "unit_cells": [int(x) for x in s.unit_cells], "init_cycles": init, "production_cycles": prod,
            "seeds": SEEDS, "runs": runs,
            "loading_mean": float(L.mean()), "loading_se": float(L.std(ddof=1) / np.sqrt(len(L))),
            "enthalpy_mean_K": float(H.mean()), "enthalpy_se_K": float(H.std(ddof=1) / np.sqrt(len(H))),
            "source": "reference simulate (oracle/_ref) built from the reference sources",
        }
        if name in IDEAL:
            doc["ideal_gas_rosenbluth_reference"], doc["ideal_gas_rosenbluth_reference_err"] = IDEAL[name]
        with open(os.path.join(OUT, f"stat_{name}.json"), "w") as fh:
            json.dump(doc, fh, indent=1)
        print(name, doc["loading_mean"], "+-", doc["loading_se"], doc["enthalpy_mean_K"], "+-", doc["enthalpy_se_K"])


if __name__ == "__main__":
    main(sys.argv[1:])
