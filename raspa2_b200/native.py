"""ctypes binding of libraspa_gpu.so (include/raspa_gpu.h).

The library is the product: there is no CPU fallback. Loading fails loudly
when the shared object is missing or cannot be loaded, and creating a system
fails when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import build as _build
from . import units
from .systems import System, kvector_indices

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

RGPU_FP64 = 0
RGPU_MIXED = 1
RGPU_MIXED_CC64 = 2   # mixed, with FP64 distances, real-space charge-charge terms and dS(k) (engine only)
RGPU_E_INVALID = -1   # include/raspa_gpu.h
RGPU_FRAMEWORK_FULL = 0
RGPU_FRAMEWORK_GRID = 1

EXPORTS = [
    "rgpu_error_string", "rgpu_device_count", "rgpu_system_create", "rgpu_system_destroy",
    "rgpu_set_adsorbates", "rgpu_get_adsorbates", "rgpu_update_molecule", "rgpu_insert_molecule",
    "rgpu_remove_molecule", "rgpu_bead_energies", "rgpu_move_energy_difference",
    "rgpu_ewald_fourier_difference", "rgpu_ewald_accept", "rgpu_total_energy", "rgpu_grid_build",
    "rgpu_grid_interpolate", "rgpu_engine_create", "rgpu_engine_destroy", "rgpu_engine_run",
    "rgpu_engine_sync", "rgpu_system_state", "rgpu_system_set_energy", "rgpu_fp32_peak_probe",
    "rgpu_engine_cluster", "rgpu_grid_interpolate_noalloc", "rgpu_system_set_limits", "rgpu_system_averages",
    "rgpu_system_reset_averages", "rgpu_engine_use_graph", "rgpu_engine_create_ex", "rgpu_engine_set_split", "rgpu_intra_energy",
    "rgpu_system_set_grids", "rgpu_system_checkpoint_size", "rgpu_system_checkpoint", "rgpu_system_restore",
    "rgpu_grid_build_coulomb", "rgpu_system_set_coulomb_grid", "rgpu_engine_get_state", "rgpu_engine_set_adsorbates",
    "rgpu_engine_staging_bytes", "rgpu_engine_replace_system", "rgpu_system_set_framework_model",
    "rgpu_grid_read_file_header", "rgpu_grid_read_file", "rgpu_grid_write_file", "rgpu_grid_file_path",
]

RGPU_NOALLOC_MAX_POINTS = 8192   # include/raspa_gpu.h


class SystemDesc(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3), ("cutoff", C.c_double), ("beta", C.c_double),
        ("coulomb", C.c_double), ("overlap", C.c_double),
        ("nfw", C.c_int), ("fw_xyz", _dp), ("fw_type", _ip), ("fw_q", _dp),
        ("ntypes", C.c_int), ("eps", _dp), ("sig2", _dp), ("shift", _dp),
        ("natom", C.c_int), ("mol_type", _ip), ("mol_q", _dp), ("mol_ref", _dp),
        ("start_bead", C.c_int), ("ewald", C.c_int), ("alpha", C.c_double),
        ("kmax", C.c_int * 3), ("maxmol", C.c_int),
        ("move_cum", C.c_double * 6), ("max_translation", C.c_double),
        ("max_rotation", C.c_double), ("fugacity_beta_v", C.c_double),
        ("ntrial_first", C.c_int), ("ntrial", C.c_int),
        ("seed", C.c_uint64), ("stream_id", C.c_uint32),
        ("flexible", C.c_int), ("bond", C.c_double), ("bend_k", C.c_double), ("bend_theta0", C.c_double),
        ("torsion", C.c_double * 4), ("chain_scheme", C.c_int), ("ntors", C.c_int),
        ("cell_matrix", C.c_double * 9),
    ]


class NativeError(RuntimeError):
    pass


_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_stale: bool = True):
    """Loads libraspa_gpu.so (building it in-tree first if it is stale and
    nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_stale and _build.stale():
        try:
            _build.build()
        except Exception as e:  # no toolchain: only a prebuilt library can be used
            if not os.path.exists(path):
                raise NativeError(f"libraspa_gpu.so is missing and could not be built: {e}")
    if not os.path.exists(path):
        raise NativeError(f"libraspa_gpu.so not found at {path}")
    L = C.CDLL(path)
    L.rgpu_error_string.restype = C.c_char_p
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        msg = load().rgpu_error_string(rc)
        raise NativeError(f"libraspa_gpu error {rc}: {msg.decode() if msg else ''}")


def device_count() -> int:
    return int(load().rgpu_device_count())


def fp32_peak_tflops() -> float:
    """Measured FP32 FMA throughput of the current device (TFLOP/s)."""
    t = C.c_double()
    s = C.c_double()
    _check(load().rgpu_fp32_peak_probe(C.byref(t), C.byref(s)))
    return t.value


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class GpuSystem:
    """One simulation box on the GPU (handle of rgpu_system)."""

    def __init__(self, sysm: System, maxmol: int = 512, seed: int = 12345, stream_id: int = 0,
                 max_translation: Optional[float] = None, max_rotation: Optional[float] = None):
        L = load()
        self.sysm = sysm
        self.init_args = dict(maxmol=maxmol, seed=seed, stream_id=stream_id, max_translation=max_translation,
                              max_rotation=max_rotation)
        eps, sig2, shift = sysm.lj_tables()
        pos, t, q = sysm.framework()
        keep = []

        def k(a, dt):
            a = _arr(a, dt)
            keep.append(a)
            return a

        d = SystemDesc()
        d.box[:] = [float(x) for x in sysm.box]
        if sysm.triclinic:
            d.cell_matrix[:] = [float(x) for x in sysm.box_matrix.reshape(-1)]
        d.cutoff = sysm.cutoff
        d.beta = units.beta(sysm.temperature)
        d.coulomb = units.COULOMBIC_CONVERSION_FACTOR
        d.overlap = units.ENERGY_OVERLAP_CRITERIA
        fwx = k(pos, np.float64); fwt = k(t, np.int32); fwq = k(q, np.float64)
        d.nfw = len(fwt)
        d.fw_xyz = fwx.ctypes.data_as(_dp); d.fw_type = fwt.ctypes.data_as(_ip); d.fw_q = fwq.ctypes.data_as(_dp)
        e = k(eps, np.float64); s2 = k(sig2, np.float64); sh = k(shift, np.float64)
        d.ntypes = e.shape[0]
        d.eps = e.ctypes.data_as(_dp); d.sig2 = s2.ctypes.data_as(_dp); d.shift = sh.ctypes.data_as(_dp)
        mt = k(sysm.molecule_types(), np.int32); mq = k(sysm.molecule.charges(), np.float64)
        mr = k(sysm.molecule.positions, np.float64)
        d.natom = len(mt)
        d.mol_type = mt.ctypes.data_as(_ip); d.mol_q = mq.ctypes.data_as(_dp); d.mol_ref = mr.ctypes.data_as(_dp)
        d.start_bead = sysm.molecule.starting_bead
        d.ewald = 1 if sysm.ewald else 0
        d.alpha = sysm.alpha
        d.kmax[:] = list(sysm.kmax)
        d.maxmol = maxmol
        d.move_cum[:] = list(sysm.moves.cumulative())
        d.max_translation = sysm.max_translation if max_translation is None else max_translation
        d.max_rotation = (np.deg2rad(sysm.max_rotation_deg) if max_rotation is None else max_rotation)
        d.fugacity_beta_v = (units.beta(sysm.temperature) * units.pressure_to_internal(sysm.pressure)
                             * sysm.volume / sysm.ideal_gas_rosenbluth)
        d.ntrial_first = sysm.trials_first_bead
        d.ntrial = sysm.trials
        d.seed = seed
        d.stream_id = stream_id
        mol = sysm.molecule
        if not mol.rigid:
            d.flexible = 1
            d.bond = mol.bond
            d.bend_k = mol.bend_k * units.KELVIN_TO_ENERGY
            d.bend_theta0 = np.deg2rad(mol.bend_theta0)
            d.torsion[:] = [t * units.KELVIN_TO_ENERGY for t in mol.torsion]
            d.chain_scheme = sysm.chain_scheme
            d.ntors = sysm.torsion_trials
        self.natom = d.natom
        self.maxmol = maxmol
        h = C.c_void_p()
        _check(L.rgpu_system_create(C.byref(h), C.byref(d)))
        self.h = h
        self.nk = len(kvector_indices(sysm.kmax)) if sysm.ewald else 0

    def close(self):
        if getattr(self, "h", None):
            load().rgpu_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state ------------------------------------------------------------
    def set_adsorbates(self, xyz):
        xyz = _arr(np.asarray(xyz, float).reshape(-1, self.natom, 3), np.float64)
        _check(load().rgpu_set_adsorbates(self.h, len(xyz), xyz.ctypes.data_as(_dp)))

    def adsorbates(self) -> np.ndarray:
        n = C.c_int()
        _check(load().rgpu_get_adsorbates(self.h, C.byref(n), None, 0))
        out = np.zeros((max(n.value, 1), self.natom, 3))
        _check(load().rgpu_get_adsorbates(self.h, C.byref(n), out.ctypes.data_as(_dp), out.shape[0]))
        return out[: n.value]

    def update_molecule(self, m, xyz):
        x = _arr(xyz, np.float64)
        _check(load().rgpu_update_molecule(self.h, C.c_int(m), x.ctypes.data_as(_dp)))

    def insert_molecule(self, xyz):
        x = _arr(xyz, np.float64)
        _check(load().rgpu_insert_molecule(self.h, x.ctypes.data_as(_dp)))

    def remove_molecule(self, m):
        _check(load().rgpu_remove_molecule(self.h, C.c_int(m)))

    # ---- energies -----------------------------------------------------------
    def bead_energies(self, xyz, atom, exclude, precision=RGPU_FP64) -> np.ndarray:
        x = _arr(np.asarray(xyz, float).reshape(-1, 3), np.float64)
        n = len(x)
        a = _arr(np.broadcast_to(atom, (n,)), np.int32)
        e = _arr(np.broadcast_to(exclude, (n,)), np.int32)
        out = np.zeros((n, 4))
        _check(load().rgpu_bead_energies(self.h, C.c_int(precision), C.c_int(n), x.ctypes.data_as(_dp),
                                         a.ctypes.data_as(_ip), e.ctypes.data_as(_ip), out.ctypes.data_as(_dp)))
        return out

    def move_difference(self, m, new_xyz, precision=RGPU_FP64):
        x = _arr(new_xyz, np.float64)
        out = np.zeros(4)
        ov = C.c_int()
        _check(load().rgpu_move_energy_difference(self.h, C.c_int(precision), C.c_int(m), x.ctypes.data_as(_dp),
                                                  out.ctypes.data_as(_dp), C.byref(ov)))
        return bool(ov.value), out

    def ewald_difference(self, old_mol=-1, new_xyz=None, precision=RGPU_FP64):
        out = np.zeros(3)
        x = None if new_xyz is None else _arr(new_xyz, np.float64)
        _check(load().rgpu_ewald_fourier_difference(self.h, C.c_int(precision), C.c_int(old_mol),
                                                    None if x is None else x.ctypes.data_as(_dp),
                                                    out.ctypes.data_as(_dp)))
        return out

    def ewald_accept(self):
        _check(load().rgpu_ewald_accept(self.h))

    def total_energy(self) -> np.ndarray:
        out = np.zeros(6)
        _check(load().rgpu_total_energy(self.h, out.ctypes.data_as(_dp)))
        return out

    def set_grids(self, grid_ptrs, npts, size, shift, cell):
        """Host VDW energies of the engine from energy grids: grid_ptrs[a] is
        the device pointer of the grid of molecule atom a (rgpu_system_set_grids);
        None switches them off."""
        L = load()
        self.grids_active = grid_ptrs is not None
        if grid_ptrs is None:
            _check(L.rgpu_system_set_grids(self.h, None, None, None, None, None))
            return
        arr = (C.c_void_p * len(grid_ptrs))(*grid_ptrs)
        n = _arr(npts, np.int32); s = _arr(size, np.float64); sh = _arr(shift, np.float64); ce = _arr(cell, np.float64)
        _check(L.rgpu_system_set_grids(self.h, arr, n.ctypes.data_as(_ip), s.ctypes.data_as(_dp),
                                       sh.ctypes.data_as(_dp), ce.ctypes.data_as(_dp)))

    def set_framework_model(self, model: int):
        """RGPU_FRAMEWORK_GRID: the per-call energies (bead_energies,
        move_difference, total_energy) take the framework terms from the grids,
        as the reference's GRID framework model; RGPU_FRAMEWORK_FULL (the
        default) sums the framework pairs."""
        _check(load().rgpu_system_set_framework_model(self.h, C.c_int(model)))

    def use_energy_grids(self, spacing: float, like: Optional["GpuSystem"] = None):
        """Builds one energy grid per pseudo-atom type of the molecule over the
        unit cell (a triclinic cell: over its enclosing box), int(size / spacing) intervals per axis,
        made odd, as MakeGrid counts them from SpacingVDWGrid
        (src/grids.c:486-492), in device memory
        this object keeps, and switches the engine's host VDW energies to
        them. With `like` (a system of the same framework and molecule whose
        grids are built at this spacing) its grids are shared instead of
        built. Returns the grid geometry (npts, size, shift, cell)."""
        import torch
        uc = np.asarray(self.sysm.unit_cell, float)
        if self.sysm.triclinic:
            # the enclosing box of the unit cell (src/grids.c:336-360)
            m = self.sysm.unit_cell_matrix
            size = np.abs(m).sum(axis=1)
            shift = np.minimum(m, 0.0).sum(axis=1)
        else:
            size = uc
            shift = np.zeros(3)
        npts = (size / spacing).astype(np.int32)
        npts += npts % 2 == 0
        n = int(np.prod(npts.astype(np.int64) + 1)) * 8
        types = [int(t) for t in self.sysm.molecule_types()]
        if like is not None:
            o = like.sysm
            if not (np.array_equal(o.unit_cell, self.sysm.unit_cell) and np.array_equal(o.frac, self.sysm.frac)
                    and list(o.uc_types) == list(self.sysm.uc_types) and like._grid_geom[0].tolist() == npts.tolist()
                    and o.molecule.atom_types == self.sysm.molecule.atom_types):
                raise ValueError("grids can be shared only between systems of one framework, molecule and spacing")
            self.share_grids_of(like)
            return self._grid_geom
        else:
            bufs = {}
            for t in sorted(set(types)):
                buf = torch.empty(n, dtype=torch.float32, device="cuda")
                torch.cuda.synchronize()
                self.grid_build(t, npts, size, shift, buf.data_ptr())
                bufs[t] = buf
            if np.any(self.sysm.molecule.charges() != 0.0):
                # the Coulomb grid: odd point counts as well (src/grids.c:588-594)
                nc = npts.copy()
                buf = torch.empty(int(np.prod(nc.astype(np.int64) + 1)) * 8, dtype=torch.float32, device="cuda")
                torch.cuda.synchronize()
                self.grid_build_coulomb(nc, size, shift, buf.data_ptr())
                bufs["coulomb"] = (buf, nc)
        self._grids = bufs
        self._grid_geom = (npts, size, shift, uc)
        self._apply_grids()
        return self._grid_geom

    def _apply_grids(self):
        types = [int(t) for t in self.sysm.molecule_types()]
        npts, size, shift, cell = self._grid_geom
        if "coulomb" in self._grids:
            buf, nc = self._grids["coulomb"]
            self.set_coulomb_grid(buf.data_ptr(), nc, size, shift, cell)
        self.set_grids([self._grids[t].data_ptr() for t in types], npts, size, shift, cell)

    def share_grids_of(self, other: "GpuSystem"):
        """Uses the grids `other` uses (a system of the same framework and
        molecule)."""
        self._grids = other._grids
        self._grid_geom = other._grid_geom
        self._apply_grids()

    def intra_energy(self) -> float:
        """Intramolecular energy of flexible chains (rgpu_intra_energy)."""
        out = C.c_double()
        _check(load().rgpu_intra_energy(self.h, C.byref(out)))
        return out.value

    def state(self):
        e = np.zeros(8)
        c = np.zeros(20, np.int64)
        n = C.c_int()
        st = C.c_int()
        step = C.c_ulonglong()
        _check(load().rgpu_system_state(self.h, e.ctypes.data_as(_dp), c.ctypes.data_as(C.POINTER(C.c_longlong)),
                                        C.byref(n), C.byref(st), C.byref(step)))
        return {"energy": e, "counters": c, "nmol": n.value, "status": st.value, "step": step.value}

    def set_limits(self, end_step: int = 0, avg_start: int = 0):
        """The engine stops advancing this system at step `end_step`
        (exclusive, 0 = never) and samples averages from `avg_start` on."""
        _check(load().rgpu_system_set_limits(self.h, C.c_ulonglong(end_step), C.c_ulonglong(avg_start)))

    def averages(self) -> dict:
        """Ensemble averages over the sampled steps: loading <N>, energy <U>
        (internal units), enthalpy of adsorption (internal units, from the
        N-U fluctuation formula) and the raw sums."""
        sm = np.zeros(8)
        _check(load().rgpu_system_averages(self.h, sm.ctypes.data_as(_dp)))
        n = max(sm[0], 1.0)
        N, N2, U, UN = sm[1] / n, sm[2] / n, sm[3] / n, sm[4] / n
        var = N2 - N * N
        kT = units.K_B * self.sysm.temperature
        dh = (UN - U * N) / var - kT if var > 0 else float("nan")
        widom = sm[6] / sm[7] if sm[7] > 0 else float("nan")
        return {"samples": int(sm[0]), "loading": N, "energy": U, "enthalpy": dh, "widom_weight": widom,
                "sums": sm}

    def checkpoint(self) -> bytes:
        """The system's whole mutable state (rgpu_system_checkpoint)."""
        L = load()
        n = C.c_size_t()
        _check(L.rgpu_system_checkpoint_size(self.h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(L.rgpu_system_checkpoint(self.h, buf, n))
        return buf.raw

    def restore(self, data: bytes):
        """Continues from a checkpoint of a system of the same model."""
        buf = C.create_string_buffer(bytes(data), len(data))
        _check(load().rgpu_system_restore(self.h, buf, C.c_size_t(len(data))))

    def reset_averages(self):
        _check(load().rgpu_system_reset_averages(self.h))

    def set_energy(self, e8):
        e = _arr(np.resize(np.asarray(e8, float), 8), np.float64)
        _check(load().rgpu_system_set_energy(self.h, e.ctypes.data_as(_dp)))

    # ---- grids --------------------------------------------------------------
    def grid_build_coulomb(self, npts, size, shift, d_grid_ptr: int):
        n = _arr(npts, np.int32); s = _arr(size, np.float64); sh = _arr(shift, np.float64)
        _check(load().rgpu_grid_build_coulomb(self.h, n.ctypes.data_as(_ip), s.ctypes.data_as(_dp),
                                              sh.ctypes.data_as(_dp), C.c_void_p(d_grid_ptr)))

    def set_coulomb_grid(self, d_grid_ptr, npts=None, size=None, shift=None, cell=None):
        """rgpu_system_set_coulomb_grid; None removes it."""
        L = load()
        if d_grid_ptr is None:
            _check(L.rgpu_system_set_coulomb_grid(self.h, None, None, None, None, None))
            return
        n = _arr(npts, np.int32); s = _arr(size, np.float64); sh = _arr(shift, np.float64); ce = _arr(cell, np.float64)
        _check(L.rgpu_system_set_coulomb_grid(self.h, C.c_void_p(d_grid_ptr), n.ctypes.data_as(_ip),
                                              s.ctypes.data_as(_dp), sh.ctypes.data_as(_dp), ce.ctypes.data_as(_dp)))

    def grid_build(self, type_: int, npts, size, shift, d_grid_ptr: int):
        n = _arr(npts, np.int32); s = _arr(size, np.float64); sh = _arr(shift, np.float64)
        _check(load().rgpu_grid_build(self.h, C.c_int(type_), n.ctypes.data_as(_ip), s.ctypes.data_as(_dp),
                                      sh.ctypes.data_as(_dp), C.c_void_p(d_grid_ptr)))


def grid_interpolate(d_grid_ptr: int, npts, size, shift, cell, xyz) -> np.ndarray:
    n = _arr(npts, np.int32); s = _arr(size, np.float64); sh = _arr(shift, np.float64)
    ce = _arr(cell, np.float64)
    x = _arr(np.asarray(xyz, float).reshape(-1, 3), np.float64)
    out = np.zeros(len(x))
    _check(load().rgpu_grid_interpolate(C.c_void_p(d_grid_ptr), n.ctypes.data_as(_ip), s.ctypes.data_as(_dp),
                                        sh.ctypes.data_as(_dp), ce.ctypes.data_as(_dp), C.c_int(len(x)),
                                        x.ctypes.data_as(_dp), out.ctypes.data_as(_dp)))
    return out


def grid_interpolate_noalloc(d_grid_ptr: int, npts, size, shift, cell, xyz) -> np.ndarray:
    """rgpu_grid_interpolate_noalloc: as grid_interpolate, through the
    library's static device scratch (at most RGPU_NOALLOC_MAX_POINTS points,
    no device allocation; overlapping calls on one device race)."""
    n = _arr(npts, np.int32); s = _arr(size, np.float64); sh = _arr(shift, np.float64)
    ce = _arr(cell, np.float64)
    x = _arr(np.asarray(xyz, float).reshape(-1, 3), np.float64)
    out = np.zeros(len(x))
    _check(load().rgpu_grid_interpolate_noalloc(C.c_void_p(d_grid_ptr), n.ctypes.data_as(_ip),
                                                s.ctypes.data_as(_dp), sh.ctypes.data_as(_dp),
                                                ce.ctypes.data_as(_dp), C.c_int(len(x)), x.ctypes.data_as(_dp),
                                                out.ctypes.data_as(_dp)))
    return out


class GridFileHeader(C.Structure):
    """rgpu_grid_file_header: the header of the reference's grid files
    (src/grids.c:726-732; the Coulomb file adds the Ewald precision)."""
    _fields_ = [("spacing", C.c_double), ("npts", C.c_int * 3), ("size", C.c_double * 3),
                ("shift", C.c_double * 3), ("delta", C.c_double * 3), ("unit_cell", C.c_double * 3),
                ("unit_cells", C.c_int * 3), ("ewald_precision", C.c_double)]

    def as_dict(self) -> dict:
        return {"spacing": self.spacing, "n": list(self.npts), "size": list(self.size), "shift": list(self.shift),
                "delta": list(self.delta), "cell": list(self.unit_cell), "ncell": list(self.unit_cells),
                "ewald_precision": self.ewald_precision}

    @classmethod
    def of(cls, meta: dict) -> "GridFileHeader":
        h = cls()
        h.spacing = meta["spacing"]
        h.npts[:] = [int(x) for x in meta["n"]]
        h.size[:] = [float(x) for x in meta["size"]]
        h.shift[:] = [float(x) for x in meta["shift"]]
        h.delta[:] = [float(x) for x in meta["delta"]]
        h.unit_cell[:] = [float(x) for x in meta["cell"]]
        h.unit_cells[:] = [int(x) for x in meta["ncell"]]
        h.ewald_precision = float(meta.get("ewald_precision", 0.0))
        return h


def grid_file_header(path: str, coulomb: bool = False) -> GridFileHeader:
    """The header of a reference grid file (checked against the file size)."""
    h = GridFileHeader()
    _check(load().rgpu_grid_read_file_header(os.fsencode(path), C.c_int(int(coulomb)), C.byref(h)))
    return h


def grid_read_file(path: str, d_grid_ptr: int, capacity: int, coulomb: bool = False) -> GridFileHeader:
    """Reads a reference grid file into device memory (point-major layout);
    capacity in floats."""
    h = GridFileHeader()
    _check(load().rgpu_grid_read_file(os.fsencode(path), C.c_int(int(coulomb)), C.byref(h), C.c_void_p(d_grid_ptr),
                                      C.c_size_t(capacity)))
    return h


def grid_write_file(path: str, header: GridFileHeader, d_grid_ptr: int, coulomb: bool = False):
    """Writes a device grid to `path` in the reference's file format."""
    _check(load().rgpu_grid_write_file(os.fsencode(path), C.c_int(int(coulomb)), C.byref(header),
                                       C.c_void_p(d_grid_ptr)))


def grid_file_path(raspa_dir: str, forcefield: str, framework: str, spacing: float,
                   pseudo_atom: Optional[str] = None, shifted: bool = True, unit_cells=None) -> str:
    """The reference's path of a VDW grid file (pseudo_atom given) or of the
    Ewald Coulomb grid file (pseudo_atom None, unit_cells given)."""
    buf = C.create_string_buffer(4096)
    uc = None if unit_cells is None else (C.c_int * 3)(*[int(x) for x in unit_cells])
    _check(load().rgpu_grid_file_path(buf, C.c_size_t(len(buf)), os.fsencode(raspa_dir), os.fsencode(forcefield),
                                      os.fsencode(framework), C.c_double(spacing),
                                      None if pseudo_atom is None else os.fsencode(pseudo_atom),
                                      C.c_int(int(shifted)), uc))
    return buf.value.decode()


class Engine:
    """Persistent batched engine over several GpuSystems (rgpu_engine)."""

    def __init__(self, systems: Sequence[GpuSystem], precision=RGPU_MIXED, threads=512, cluster=0, ctas_per_sm=1):
        L = load()
        arr = (C.c_void_p * len(systems))(*[s.h for s in systems])
        h = C.c_void_p()
        _check(L.rgpu_engine_create_ex(C.byref(h), arr, C.c_int(len(systems)), C.c_int(precision), C.c_int(threads),
                                       C.c_int(cluster), C.c_int(ctas_per_sm)))
        self.ctas_per_sm = ctas_per_sm
        self.cluster = int(L.rgpu_engine_cluster(h))
        self.threads = threads
        self.precision = precision
        self.h = h
        self.systems = list(systems)
        self.split = ([], 0)

    def run(self, nsteps: int, stream: Optional[int] = None):
        _check(load().rgpu_engine_run(self.h, C.c_longlong(nsteps), C.c_void_p(stream or 0)))

    def sync(self):
        _check(load().rgpu_engine_sync(self.h))

    def get_states(self, positions: bool = True):
        """Every system's state (and positions) with one transfer
        (rgpu_engine_get_state): a list of dicts as GpuSystem.state(), with
        "xyz" [nmol, natom, 3] when positions is true (a view of a buffer
        that the next call overwrites: copy it to keep it)."""
        n = len(self.systems)
        e = np.zeros((n, 8)); c = np.zeros((n, 20), np.int64)
        nm = np.zeros(n, np.int32); stt = np.zeros(n, np.int32); stp = np.zeros(n, np.uint64)
        bufs, ptrs = None, None
        if positions:
            if getattr(self, "_xyz_bufs", None) is None:
                self._xyz_bufs = [np.zeros((g.init_args["maxmol"], g.natom, 3)) for g in self.systems]
                self._xyz_ptrs = (C.POINTER(C.c_double) * n)(*[b.ctypes.data_as(_dp) for b in self._xyz_bufs])
            bufs, ptrs = self._xyz_bufs, self._xyz_ptrs
        _check(load().rgpu_engine_get_state(self.h, e.ctypes.data_as(_dp), c.ctypes.data_as(C.POINTER(C.c_longlong)),
                                            nm.ctypes.data_as(_ip), stt.ctypes.data_as(_ip),
                                            stp.ctypes.data_as(C.POINTER(C.c_ulonglong)), ptrs))
        out = []
        for i in range(n):
            d = {"energy": e[i], "counters": c[i], "nmol": int(nm[i]), "status": int(stt[i]), "step": int(stp[i])}
            if positions:
                d["xyz"] = bufs[i][: nm[i]]
            out.append(d)
        return out

    def set_adsorbates(self, xyz_list):
        """Every system's configuration with one transfer
        (rgpu_engine_set_adsorbates); xyz_list[i]: [nmol, natom, 3]."""
        n = len(self.systems)
        keep = [np.ascontiguousarray(np.asarray(x, float).reshape(-1, g.natom, 3))
                for x, g in zip(xyz_list, self.systems)]
        nm = np.array([len(x) for x in keep], np.int32)
        ptrs = (C.POINTER(C.c_double) * n)(*[x.ctypes.data_as(_dp) for x in keep])
        _check(load().rgpu_engine_set_adsorbates(self.h, nm.ctypes.data_as(_ip), ptrs))

    def staging_bytes(self) -> int:
        n = C.c_size_t()
        _check(load().rgpu_engine_staging_bytes(self.h, C.byref(n)))
        return n.value

    def set_split(self, second: Sequence[int], cluster_b: int):
        """Run the systems at indices `second` in a second launch with
        clusters of `cluster_b` CTAs, beside the first (rgpu_engine_set_split);
        an empty `second` returns to one launch."""
        idx = [int(i) for i in second]
        arr = (C.c_int * max(len(idx), 1))(*idx)
        _check(load().rgpu_engine_set_split(self.h, arr, C.c_int(len(idx)), C.c_int(cluster_b)))
        self.split = (idx, int(cluster_b) if idx else 0)

    def use_graph(self, on: bool = True):
        """Replay a CUDA graph of the launch in run() (rgpu_engine_use_graph)."""
        _check(load().rgpu_engine_use_graph(self.h, C.c_int(1 if on else 0)))

    def replace(self, i: int, system: GpuSystem, stream: Optional[int] = None) -> bool:
        """Puts `system` in place of system i, ordered on `stream` after the
        queued launches (rgpu_engine_replace_system). Returns False when the
        system does not fit this engine's layout (build a new engine)."""
        rc = load().rgpu_engine_replace_system(self.h, C.c_int(i), system.h, C.c_void_p(stream or 0))
        if rc == RGPU_E_INVALID:
            return False
        _check(rc)
        self.systems[i] = system
        return True

    def close(self):
        if getattr(self, "h", None):
            load().rgpu_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
