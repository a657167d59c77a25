"""Loads the committed golden fixtures and rebuilds their systems."""
import json
import os

import numpy as np

from raspa2_b200 import systems

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

BUILDERS = {
    "co2_tiny": lambda seed: systems.tiny_co2_system(),
    "co2_config1": lambda seed: systems.co2_system(seed=seed),
    "methane_config0": lambda seed: systems.methane_system(seed=seed),
    "co2_triclinic": lambda seed: systems.co2_triclinic_system(seed=seed),
}
ENERGY_CASES = list(BUILDERS)


def load(name):
    with open(os.path.join(HERE, f"{name}.json")) as fh:
        return json.load(fh)


def system_of(case):
    b = case["system"]["builder"]
    if b == "methane_222":
        s = systems.methane_system(seed=case["system"]["seed"])
        s.unit_cells = np.array([2, 2, 2])
        return s
    return BUILDERS[b](case["system"]["seed"])
