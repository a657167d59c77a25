"""Generates tests/golden/restart_<case>.txt and restart_<case>.json: a
restart file written by the reference program, and the energies it printed
for that same configuration.

Runs in the build container only (it needs oracle/_ref/simulate, built from
the reference's sources by `make -C oracle ref`). Each case runs the
reference briefly from an empty framework. At the end of a run the reference
prints its "Current (full final energy) Energy Status" (a full recomputation)
and then writes the restart file of the final configuration
(src/monte_carlo.c:1040-1044), so the two describe the same molecules. The
.txt is the reference's restart file as written; the .json holds that
energy block in K and the state point.

    python tests/golden/make_restart_golden.py [case ...]
"""
from __future__ import annotations

import dataclasses
import glob
import json
import os
import shutil
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from raspa2_b200 import output, raspa_io, systems  # noqa: E402

SIMULATE = os.path.join(ROOT, "oracle", "_ref", "simulate")
OUT = os.path.dirname(os.path.abspath(__file__))

# name -> (builder, state point, initialisation cycles, production cycles, seed)
CASES = {
    "co2_config1": (lambda: systems.co2_system(seed=1), dict(pressure=1e5, temperature=298.0), 4, 2, 611),
    "hexane_small": (lambda: systems.hexane_system(seed=4, n_atoms=1200, cell=26.0),
                     dict(pressure=1e6, temperature=433.0), 15, 5, 612),
}


def run_case(name, work):
    build, state, init, prod, seed = CASES[name]
    s = dataclasses.replace(build(), **state)
    d = os.path.join(work, name)
    raspa_io.write_inputs(s, d, cycles=prod, init_cycles=init, print_every=10 ** 9, seed=seed)
    r = subprocess.run([SIMULATE, "-i", "simulation.input"], cwd=d, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"simulate failed in {d}: {r.stderr[-500:]}")
    data = glob.glob(os.path.join(d, "Output", "System_0", "*.data"))[0]
    energies = output.parse_energy_status(open(data).read(), "full final energy")
    rst = glob.glob(os.path.join(d, "Restart", "System_0", "restart_*"))[0]
    shutil.copyfile(rst, os.path.join(OUT, f"restart_{name}.txt"))
    meta = {"case": name, "system": s.name, "pressure_Pa": s.pressure, "temperature_K": s.temperature,
            "restart_file_name": os.path.basename(rst), "energies_K": energies,
            "source": "reference simulate (oracle/_ref) built from the reference sources; "
                      f"{init} initialisation + {prod} production cycles from empty, seed {seed}"}
    with open(os.path.join(OUT, f"restart_{name}.json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    print(name, len(open(rst).read().splitlines()), "lines")


def main(argv):
    work = tempfile.mkdtemp(prefix="raspa_restart_")
    try:
        for name in argv or list(CASES):
            run_case(name, work)
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main(sys.argv[1:])
