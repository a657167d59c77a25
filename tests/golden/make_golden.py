"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs in the build container only (it needs the reference sources and the
harness built by `make -C oracle ref`): each case writes a seeded synthetic
system as RASPA input files, drives oracle/_ref/ref_harness (the reference's
own energy, Ewald, CBMC and grid routines) and stores inputs and outputs as
small JSON files. The committed JSON is what the tests read; nothing at test
time needs the reference.

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py coulomb    # only grid_co2_coulomb.json
    python tests/golden/make_golden.py gridfiles  # only grid_co2_files.json + grid_files/
    python tests/golden/make_golden.py triclinic  # only co2_triclinic.json
    python tests/golden/make_golden.py gridtri    # only grid_co2_triclinic.json
"""
from __future__ import annotations

import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from raspa2_b200 import raspa_io, systems  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
OUT = os.path.dirname(os.path.abspath(__file__))


def run_harness(d, cmds):
    with open(os.path.join(d, "cmds"), "w") as fh:
        fh.write("\n".join(cmds) + "\n")
    r = subprocess.run([HARNESS, d, os.path.join(d, "cmds"), os.path.join(d, "out")],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"harness failed ({r.returncode}): {r.stderr[-2000:]}")
    rows = []
    with open(os.path.join(d, "out")) as fh:
        for line in fh:
            p = line.split()
            rows.append(p)
    return rows


def fmt(v):
    return " ".join(f"{x:.17g}" for x in np.asarray(v, float).reshape(-1))


def random_molecule(rng, sysm, fw, min_d=2.2):
    """A randomly oriented molecule away from framework atoms."""
    ref = sysm.molecule.positions
    sb = sysm.molecule.starting_bead
    for _ in range(10000):
        c = sysm.box_point(rng.random(3))
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, cc, d = q
        R = np.array([[a*a+b*b-cc*cc-d*d, 2*(b*cc-a*d), 2*(b*d+a*cc)],
                      [2*(b*cc+a*d), a*a-b*b+cc*cc-d*d, 2*(cc*d-a*b)],
                      [2*(b*d-a*cc), 2*(cc*d+a*b), a*a-b*b-cc*cc+d*d]])
        x = c + (ref - ref[sb]) @ R.T
        dd = sysm.min_image(x[:, None, :] - fw[None, :, :])
        if np.min(np.linalg.norm(dd, axis=2)) > min_d:
            return x
    raise RuntimeError("could not place a molecule")


def names_of(rows):
    return {int(r[1]): r[2] for r in rows if r[0] == "pseudo"}


def energy_case(name, sysm, n_mol, seed, n_points=12, n_moves=8, n_cbmc=4):
    rng = np.random.default_rng(seed)
    fw, _, _ = sysm.framework()
    mols = [random_molecule(rng, sysm, fw) for _ in range(n_mol)]
    na = sysm.molecule.n_atoms
    with tempfile.TemporaryDirectory() as d:
        raspa_io.write_inputs(sysm, d)
        cmds = ["system"] + [f"insert {fmt(m)}" for m in mols] + ["energy"]
        # bead energies at points, for every bead type of the molecule
        pts = []
        for i in range(n_points):
            p = sysm.box_point(rng.random(3))
            a = int(rng.integers(0, na))
            excl = int(rng.integers(-1, n_mol)) if n_mol else -1
            pts.append((a, p, excl))
        # a point right on a framework atom neighbourhood (overlap regime)
        pts.append((0, fw[3] + np.array([0.3, 0.0, 0.0]), -1))
        # moves: translations (some large), rotations, one overlapping move
        moves = []
        for i in range(n_moves):
            if not n_mol:
                break
            m = int(rng.integers(0, n_mol))
            x = mols[m].copy()
            if i % 2 == 0:
                x = x + rng.normal(scale=0.5, size=3)
            else:
                th = rng.uniform(-0.5, 0.5)
                c = x - x[sysm.molecule.starting_bead]
                cs, sn = np.cos(th), np.sin(th)
                c = c @ np.array([[cs, -sn, 0], [sn, cs, 0], [0, 0, 1]]).T
                x = c + x[sysm.molecule.starting_bead]
            moves.append((m, x))
        if n_mol:
            m = 0
            moves.append((m, mols[m] - mols[m][0] + fw[5] + np.array([0.2, 0.1, 0.0])))
        for (a, p, excl) in pts:
            t = sysm.molecule_types()[a]
            cmds.append(f"point {t + 1} {fmt(p)} {excl}")
        for (m, x) in moves:
            cmds.append(f"move {m} {fmt(x)}")
        ins = random_molecule(rng, sysm, fw)
        if sysm.ewald:
            cmds.append(f"ewald_insert {fmt(ins)}")
            if n_mol:
                cmds.append(f"ewald_delete {n_mol - 1}")
        # accepted move then a dependent move: exercises the S(k) bookkeeping
        acc = []
        if n_mol >= 2:
            x = mols[1] + np.array([0.4, -0.3, 0.2])
            y = mols[0] + np.array([-0.2, 0.25, 0.3])
            cmds.append(f"accept 1 {fmt(x)}")
            cmds.append(f"move 0 {fmt(y)}")
            cmds.append("energy")
            acc = [(1, x), (0, y)]
        cbmc = []
        for i in range(n_cbmc):
            s = 1000 + 17 * i
            cmds.append(f"cbmc_insert {s}")
            cbmc.append(("insert", -1, s))
            if n_mol:
                m = int(rng.integers(0, n_mol))
                s2 = 5000 + 31 * i
                # the accepted move above changed molecule 1: track positions
                cmds.append(f"cbmc_delete {m} {s2}")
                cbmc.append(("delete", m, s2))
        rows = run_harness(d, cmds)
    names = names_of(rows)
    out_pts = [list(map(float, r[1:])) for r in rows if r[0] == "point"]
    out_mv = [list(map(float, r[1:])) for r in rows if r[0] == "move"]
    out_ew = [list(map(float, r[1:])) for r in rows if r[0] == "fourier"]
    out_en = [list(map(float, r[1:])) for r in rows if r[0] == "energy"]
    out_cb = [list(map(float, r[1:])) for r in rows if r[0] == "cbmc"]
    fwrows = np.array([[float(x) for x in r[1:4]] for r in rows if r[0] == "fw"])
    const = [float(x) for x in [r for r in rows if r[0] == "constants"][0][1:]]
    ewald = [float(x) for x in [r for r in rows if r[0] == "ewald"][0][1:]]
    fw_mine, _, _ = sysm.framework()
    case = {
        "name": name,
        "system": {"builder": name, "seed": int(sysm.seed)},
        "constants": const,
        "ewald": ewald,
        "pseudo_names": [names[i] for i in sorted(names)],
        "framework_max_abs_diff_vs_generator": float(np.max(np.abs(fwrows - fw_mine))),
        "n_framework": int(len(fwrows)),
        "molecules": [m.tolist() for m in mols],
        "points": [{"atom": a, "p": p.tolist(), "exclude": e, "ref": r}
                   for (a, p, e), r in zip(pts, out_pts)],
        "moves": [{"m": m, "new": x.tolist(), "ref": r} for (m, x), r in zip(moves, out_mv)],
        "insert": ins.tolist(),
        "fourier": out_ew,
        "energy": out_en,
        "accepted": [{"m": m, "new": x.tolist()} for (m, x) in acc],
        "accepted_ref": out_mv[len(moves):],
        "cbmc": [{"kind": k, "m": m, "seed": s, "ref": r} for (k, m, s), r in zip(cbmc, out_cb)],
        "trials": [sysm.trials_first_bead, sysm.trials],
    }
    return case


def read_grid_file(path):
    with open(path, "rb") as fh:
        b = fh.read()
    spacing = struct.unpack_from("d", b, 0)[0]
    n = struct.unpack_from("3i", b, 8)
    off = 8 + 12
    size = struct.unpack_from("3d", b, off); off += 24
    shift = struct.unpack_from("3d", b, off); off += 24
    delta = struct.unpack_from("3d", b, off); off += 24
    cell = struct.unpack_from("3d", b, off); off += 24
    ncell = struct.unpack_from("3i", b, off); off += 12
    npts = (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
    g = np.frombuffer(b, dtype=np.float32, count=8 * npts, offset=off).reshape(8, n[0] + 1, n[1] + 1, n[2] + 1)
    return {"spacing": spacing, "n": list(n), "size": list(size), "shift": list(shift), "delta": list(delta),
            "cell": list(cell), "ncell": list(ncell)}, g


def grid_case(seed=0, spacing=1.0):
    sysm = systems.methane_system(seed=seed)
    sysm.unit_cells = np.array([2, 2, 2])
    rng = np.random.default_rng(seed + 99)
    t = systems.TYPE_ORDER.index("CH4_sp3")
    with tempfile.TemporaryDirectory() as d:
        grid = {"types": ["CH4_sp3"], "spacing": spacing}
        raspa_io.write_inputs(sysm, d, simulation_type="MakeGrid", grid=grid)
        # the reference creates only the last levels of the grid directory
        os.makedirs(os.path.join(d, "share", "raspa", "grids"), exist_ok=True)
        # reference derivatives at sample points (CalculateDerivativesAtPositionVDW)
        pts = rng.random((10, 3)) * sysm.unit_cell
        rows = run_harness(d, [f"deriv {t + 1} {fmt(p)}" for p in pts] + ["makegrid"])
        deriv = [list(map(float, r[1:])) for r in rows if r[0] == "deriv"]
        gpath = os.path.join(d, "share", "raspa", "grids", "Local", sysm.name, f"{spacing:.6f}",
                             f"{sysm.name}_CH4_sp3_shifted.grid")
        meta, g = read_grid_file(gpath)
        # interpolation by the reference from its own grid file
        grid["use"] = True
        raspa_io.write_inputs(sysm, d, simulation_type="MonteCarlo", grid=grid)
        q = rng.random((40, 3)) * sysm.box - 0.5 * sysm.box
        rows = run_harness(d, [f"interp {t + 1} {fmt(p)}" for p in q])
        interp = [float(r[1]) for r in rows if r[0] == "interp"]
    sel = rng.integers(0, g[0].size, 64)
    flat = g.reshape(8, -1)
    return {
        "name": "grid_methane",
        "system": {"builder": "methane_222", "seed": seed},
        "meta": meta,
        "deriv_points": pts.tolist(), "deriv_ref": deriv,
        "sample_index": sel.tolist(), "sample_values": flat[:, sel].T.astype(float).tolist(),
        "plane_sums": [float(np.sum(flat[m].astype(np.float64))) for m in range(8)],
        "interp_points": q.tolist(), "interp_ref": interp,
    }


def read_coulomb_grid_file(path):
    """The Coulomb grid file (src/grids.c:856-869): the VDW header, then the
    Ewald precision, then the 8 planes."""
    with open(path, "rb") as fh:
        b = fh.read()
    spacing = struct.unpack_from("d", b, 0)[0]
    n = struct.unpack_from("3i", b, 8)
    off = 8 + 12
    size = struct.unpack_from("3d", b, off); off += 24
    shift = struct.unpack_from("3d", b, off); off += 24
    delta = struct.unpack_from("3d", b, off); off += 24
    cell = struct.unpack_from("3d", b, off); off += 24
    ncell = struct.unpack_from("3i", b, off); off += 12
    prec = struct.unpack_from("d", b, off)[0]; off += 8
    npts = (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
    g = np.frombuffer(b, dtype=np.float32, count=8 * npts, offset=off).reshape(8, n[0] + 1, n[1] + 1, n[2] + 1)
    return {"spacing": spacing, "n": list(n), "size": list(size), "shift": list(shift), "delta": list(delta),
            "cell": list(cell), "ncell": list(ncell), "ewald_precision": prec}, g


def coulomb_grid_case(seed=1, spacing=1.0):
    """The reference's Coulomb grid of the CO2 framework: derivatives at
    points, the grid file, and InterpolateCoulombGrid for the CO2 sites."""
    sysm = systems.co2_system(seed=seed)
    rng = np.random.default_rng(seed + 199)
    types = ["C_co2", "O_co2"]
    with tempfile.TemporaryDirectory() as d:
        grid = {"types": types, "spacing": spacing}
        raspa_io.write_inputs(sysm, d, simulation_type="MakeGrid", grid=grid)
        os.makedirs(os.path.join(d, "share", "raspa", "grids"), exist_ok=True)
        pts = rng.random((12, 3)) * sysm.unit_cell
        rows = run_harness(d, [f"derivreal {fmt(p)}" for p in pts] + ["makegrid"])
        deriv = [list(map(float, r[1:])) for r in rows if r[0] == "derivreal"]
        a, b, c = (int(x) for x in sysm.unit_cells)
        gpath = os.path.join(d, "share", "raspa", "grids", "Local", sysm.name, f"{spacing:.6f}", f"{a}x{b}x{c}",
                             f"{sysm.name}_Electrostatics_Ewald.grid")
        meta, g = read_coulomb_grid_file(gpath)
        grid["use"] = True
        raspa_io.write_inputs(sysm, d, simulation_type="MonteCarlo", grid=grid)
        q = rng.random((40, 3)) * sysm.box - 0.5 * sysm.box
        cmds = []
        for name in types:
            t = systems.TYPE_ORDER.index(name)
            cmds += [f"interpc {t + 1} {fmt(p)}" for p in q]
        rows = run_harness(d, cmds)
        interp = [float(r[1]) for r in rows if r[0] == "interpc"]
    sel = rng.integers(0, g[0].size, 64)
    flat = g.reshape(8, -1)
    return {
        "name": "grid_co2_coulomb",
        "system": {"builder": "co2_config1", "seed": seed},
        "meta": meta, "types": types,
        "deriv_points": pts.tolist(), "deriv_ref": deriv,
        "sample_index": sel.tolist(), "sample_values": flat[:, sel].T.astype(float).tolist(),
        "plane_sums": [float(np.sum(flat[m].astype(np.float64))) for m in range(8)],
        "plane_abs_sums": [float(np.sum(np.abs(flat[m].astype(np.float64)))) for m in range(8)],
        "interp_points": q.tolist(), "interp_ref": interp,
    }


def grid_files_case(seed=1, spacing=2.0):
    """The reference's own grid files of the CO2 framework at a coarse
    spacing (VDW grids of C_co2 and O_co2, the Ewald Coulomb grid), copied
    to tests/golden/grid_files/, with InterpolateVDWGrid and
    InterpolateCoulombGrid of the reference on those files at points."""
    import shutil
    sysm = systems.co2_system(seed=seed)
    rng = np.random.default_rng(seed + 299)
    types = ["C_co2", "O_co2"]
    dst = os.path.join(OUT, "grid_files")
    os.makedirs(dst, exist_ok=True)
    with tempfile.TemporaryDirectory() as d:
        grid = {"types": types, "spacing": spacing}
        raspa_io.write_inputs(sysm, d, simulation_type="MakeGrid", grid=grid)
        os.makedirs(os.path.join(d, "share", "raspa", "grids"), exist_ok=True)
        run_harness(d, ["makegrid"])
        base = os.path.join(d, "share", "raspa", "grids", "Local", sysm.name, f"{spacing:.6f}")
        a, b, c = (int(x) for x in sysm.unit_cells)
        files = {t: os.path.join(base, f"{sysm.name}_{t}_shifted.grid") for t in types}
        files["coulomb"] = os.path.join(base, f"{a}x{b}x{c}", f"{sysm.name}_Electrostatics_Ewald.grid")
        rel, meta = {}, {}
        for k, f in files.items():
            rel[k] = os.path.relpath(f, d)
            meta[k] = (read_coulomb_grid_file(f) if k == "coulomb" else read_grid_file(f))[0]
            shutil.copyfile(f, os.path.join(dst, os.path.basename(f)))
        grid["use"] = True
        raspa_io.write_inputs(sysm, d, simulation_type="MonteCarlo", grid=grid)
        q = rng.random((24, 3)) * sysm.box - 0.5 * sysm.box
        cmds = []
        for name in types:
            t = systems.TYPE_ORDER.index(name)
            cmds += [f"interp {t + 1} {fmt(p)}" for p in q] + [f"interpc {t + 1} {fmt(p)}" for p in q]
        rows = run_harness(d, cmds)
    vals = [float(r[1]) for r in rows if r[0] in ("interp", "interpc")]
    n = len(q)
    interp = {name: {"vdw": vals[2 * i * n: (2 * i + 1) * n], "coulomb": vals[(2 * i + 1) * n: (2 * i + 2) * n]}
              for i, name in enumerate(types)}
    return {
        "name": "grid_co2_files",
        "system": {"builder": "co2_config1", "seed": seed},
        "spacing": spacing, "types": types,
        "files": {k: os.path.basename(v) for k, v in files.items()},
        "reference_paths": rel, "meta": meta,
        "points": q.tolist(), "interp_ref": interp,
    }


def grid_triclinic_case(seed=11, spacing=1.0):
    """MakeGrid in the triclinic CO2 cell (co2_triclinic_system): the VDW
    grids of C_co2 and O_co2 and the Ewald Coulomb grid as the reference
    writes them (samples and plane sums), and the reference's
    InterpolateVDWGrid / InterpolateCoulombGrid (their TRICLINIC branches)
    at points anywhere in and around the box."""
    sysm = systems.co2_triclinic_system(seed=seed)
    rng = np.random.default_rng(seed + 399)
    types = ["C_co2", "O_co2"]
    with tempfile.TemporaryDirectory() as d:
        grid = {"types": types, "spacing": spacing}
        raspa_io.write_inputs(sysm, d, simulation_type="MakeGrid", grid=grid)
        os.makedirs(os.path.join(d, "share", "raspa", "grids"), exist_ok=True)
        run_harness(d, ["makegrid"])
        base = os.path.join(d, "share", "raspa", "grids", "Local", sysm.name, f"{spacing:.6f}")
        files = {t: os.path.join(base, f"{sysm.name}_{t}_shifted.grid") for t in types}
        files["coulomb"] = os.path.join(base, "1x1x1", f"{sysm.name}_Electrostatics_Ewald.grid")
        meta, samples, sums = {}, {}, {}
        for k, f in files.items():
            m, g = read_coulomb_grid_file(f) if k == "coulomb" else read_grid_file(f)
            flat = g.reshape(8, -1)
            sel = rng.integers(0, flat.shape[1], 64)
            meta[k] = m
            samples[k] = {"index": sel.tolist(), "values": flat[:, sel].T.astype(float).tolist()}
            sums[k] = {"sum": [float(np.sum(flat[q].astype(np.float64))) for q in range(8)],
                       "abs": [float(np.sum(np.abs(flat[q].astype(np.float64)))) for q in range(8)]}
        grid["use"] = True
        raspa_io.write_inputs(sysm, d, simulation_type="MonteCarlo", grid=grid)
        q = sysm.box_point(rng.random((24, 3)) * 1.4 - 0.2)
        cmds = []
        for name in types:
            t = systems.TYPE_ORDER.index(name)
            cmds += [f"interp {t + 1} {fmt(p)}" for p in q] + [f"interpc {t + 1} {fmt(p)}" for p in q]
        rows = run_harness(d, cmds)
    vals = [float(r[1]) for r in rows if r[0] in ("interp", "interpc")]
    n = len(q)
    interp = {name: {"vdw": vals[2 * i * n: (2 * i + 1) * n], "coulomb": vals[(2 * i + 1) * n: (2 * i + 2) * n]}
              for i, name in enumerate(types)}
    return {"name": "grid_co2_triclinic", "system": {"builder": "co2_triclinic", "seed": seed},
            "spacing": spacing, "types": types, "meta": meta, "samples": samples, "plane_sums": sums,
            "points": q.tolist(), "interp_ref": interp}


def main():
    if not os.path.exists(HARNESS):
        raise SystemExit("build the harness first: make -C oracle ref")
    if sys.argv[1:] == ["gridtri"]:
        g = grid_triclinic_case()
        with open(os.path.join(OUT, "grid_co2_triclinic.json"), "w") as fh:
            json.dump(g, fh)
        print("triclinic grids", {k: v["n"] for k, v in g["meta"].items()})
        return
    if sys.argv[1:] == ["triclinic"]:
        case = energy_case("co2_triclinic", systems.co2_triclinic_system(), 10, 14)
        with open(os.path.join(OUT, "co2_triclinic.json"), "w") as fh:
            json.dump(case, fh)
        print("co2_triclinic points", len(case["points"]), "moves", len(case["moves"]),
              "fw diff", case["framework_max_abs_diff_vs_generator"])
        return
    if sys.argv[1:] == ["gridfiles"]:
        g = grid_files_case()
        with open(os.path.join(OUT, "grid_co2_files.json"), "w") as fh:
            json.dump(g, fh)
        print("grid files", g["files"], g["meta"]["coulomb"]["n"])
        return
    if sys.argv[1:] == ["coulomb"]:
        g = coulomb_grid_case()
        with open(os.path.join(OUT, "grid_co2_coulomb.json"), "w") as fh:
            json.dump(g, fh)
        print("coulomb grid", g["meta"]["n"], len(g["interp_ref"]))
        return
    cases = {
        "co2_tiny": (systems.tiny_co2_system(), 6, 11),
        "co2_config1": (systems.co2_system(seed=1), 10, 12),
        "methane_config0": (systems.methane_system(seed=0), 8, 13),
        "co2_triclinic": (systems.co2_triclinic_system(), 10, 14),
    }
    for name, (sysm, nmol, seed) in cases.items():
        case = energy_case(name, sysm, nmol, seed)
        with open(os.path.join(OUT, f"{name}.json"), "w") as fh:
            json.dump(case, fh)
        print(name, "points", len(case["points"]), "moves", len(case["moves"]), "cbmc", len(case["cbmc"]))
    g = grid_case()
    with open(os.path.join(OUT, "grid_methane.json"), "w") as fh:
        json.dump(g, fh)
    print("grid", g["meta"]["n"], len(g["interp_ref"]))
    g = coulomb_grid_case()
    with open(os.path.join(OUT, "grid_co2_coulomb.json"), "w") as fh:
        json.dump(g, fh)
    print("coulomb grid", g["meta"]["n"], len(g["interp_ref"]))
    g = grid_files_case()
    with open(os.path.join(OUT, "grid_co2_files.json"), "w") as fh:
        json.dump(g, fh)
    print("grid files", g["files"], g["meta"]["coulomb"]["n"])


if __name__ == "__main__":
    main()
