"""Statistical parity of whole GCMC runs: the engine's average loading and
enthalpy of adsorption match the reference program's within the combined
statistical error.

The fixtures tests/golden/stat_*.json hold, per case, eight independent runs
of the reference program from an empty framework. tests/golden/make_stat_golden.py
wrote them. Here the engine runs the same system as independent replicas
(own random streams), each from empty, equilibrated, then sampled. Each
side's mean carries a standard error across its independent runs, and the
two must agree within 4 combined standard errors.

The mixed-precision engine is the form under test. Its exponents differ from
FP64 by less than 1e-3 k_B T (tests/test_gpu_parity.py), which biases
averages far below these errors.

Flexible chains (n-hexane): the fugacity term of a CBMC insertion is divided
by the molecule's ideal-gas Rosenbluth weight W_IG, which depends on how a
code draws the bonded part of its trials. The reference divides by its own
(measured by its Widom run, stored in the fixture); here the engine measures
its own W_IG by Widom insertions into an empty box, and the physical averages
must then agree.
"""
import dataclasses
import json
import os

import numpy as np
import pytest

from raspa2_b200 import native, systems, units

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NSIGMA = 4.0

# case -> (builder, replicas, equilibration steps, production steps, maxmol)
CASES = {
    "methane_config0_1e5": (lambda: systems.methane_system(seed=0), 64, 20000, 80000, 128),
    "methane_config0_1e7": (lambda: systems.methane_system(seed=0), 64, 100000, 120000, 512),
    "co2_config1_1e5": (lambda: systems.co2_system(seed=1), 64, 400000, 400000, 384),
    "hexane_small_3e4": (lambda: systems.hexane_system(seed=4, n_atoms=1200, cell=26.0), 64, 100000, 200000, 64),
}


def engine_ideal_gas_rosenbluth(molecule, temperature, nrep=64, steps=20000):
    """W_IG of `molecule` for the engine's CBMC scheme: mean Rosenbluth
    weight of Widom insertions into an empty box; (mean, standard error)."""
    s = systems.empty_box_system(molecule, temperature)
    gs = []
    for i in range(nrep):
        g = native.GpuSystem(s, maxmol=4, seed=4711 + i, stream_id=i)
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
        g.set_limits(steps, 0)
        gs.append(g)
    e = native.Engine(gs, precision=native.RGPU_MIXED)
    e.run(steps)
    e.sync()
    w = np.array([g.averages()["widom_weight"] for g in gs])
    return float(w.mean()), float(w.std(ddof=1) / np.sqrt(nrep))


def _load(case):
    with open(os.path.join(GOLDEN, f"stat_{case}.json")) as fh:
        return json.load(fh)


def engine_averages(case, pressure, temperature, ncell):
    """Per-replica average loading [molecules/unit cell] and enthalpy [K]."""
    build, nrep, equil, prod, maxmol = CASES[case]
    s = dataclasses.replace(build(), pressure=pressure, temperature=temperature)
    if not s.molecule.rigid:
        w, _ = engine_ideal_gas_rosenbluth(s.molecule, temperature)
        s = dataclasses.replace(s, ideal_gas_rosenbluth=w)
    gs = []
    for i in range(nrep):
        g = native.GpuSystem(s, maxmol=maxmol, seed=31337 + i, stream_id=i)
        g.set_adsorbates(np.zeros((0, s.molecule.n_atoms, 3)))
        g.set_limits(equil + prod, equil)
        gs.append(g)
    e = native.Engine(gs, precision=native.RGPU_MIXED)
    e.run(equil + prod)
    e.sync()
    loads, hs = [], []
    for g in gs:
        st = g.state()
        assert st["status"] == 0 and st["step"] == equil + prod
        av = g.averages()
        assert av["samples"] == prod
        loads.append(av["loading"] / ncell)
        hs.append(av["enthalpy"] / units.K_B)
    return np.array(loads), np.array(hs)


@pytest.mark.parametrize("case", sorted(CASES))
def test_averages_match_reference(cuda, case):
    ref = _load(case)
    loads, hs = engine_averages(case, ref["pressure_Pa"], ref["temperature_K"], float(np.prod(ref["unit_cells"])))
    n = len(loads)
    se_l = loads.std(ddof=1) / np.sqrt(n)
    se_h = hs.std(ddof=1) / np.sqrt(n)
    dl = abs(loads.mean() - ref["loading_mean"])
    dh = abs(hs.mean() - ref["enthalpy_mean_K"])
    assert dl <= NSIGMA * np.hypot(se_l, ref["loading_se"]), (case, loads.mean(), se_l, ref["loading_mean"],
                                                               ref["loading_se"])
    assert dh <= NSIGMA * np.hypot(se_h, ref["enthalpy_se_K"]), (case, hs.mean(), se_h, ref["enthalpy_mean_K"],
                                                                 ref["enthalpy_se_K"])
