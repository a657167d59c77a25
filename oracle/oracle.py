"""ctypes binding of the C oracle (oracle/oracle.c).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker. The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrSys(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3), ("rc2_vdw", C.c_double), ("rc2_cc", C.c_double),
        ("overlap", C.c_double), ("coulomb", C.c_double), ("beta", C.c_double),
        ("ntypes", C.c_int), ("eps", _dp), ("sig2", _dp), ("shift", _dp),
        ("nfw", C.c_int), ("fw_xyz", _dp), ("fw_type", _ip), ("fw_q", _dp),
        ("nmol", C.c_int), ("natom", C.c_int), ("maxmol", C.c_int), ("ads_xyz", _dp),
        ("mol_type", _ip), ("mol_q", _dp), ("mol_ref", _dp), ("start_bead", C.c_int),
        ("ewald", C.c_int), ("alpha", C.c_double), ("nk", C.c_int), ("kidx", _ip),
        ("kfactor", _dp), ("sk_fw", _dp), ("sk_ads", _dp),
        ("uion", C.c_double), ("net_fw", C.c_double), ("net_ads", C.c_double),
        ("flexible", C.c_int), ("bond", C.c_double), ("bend_k", C.c_double), ("bend_theta0", C.c_double),
        ("bend_sigma", C.c_double), ("torsion", C.c_double * 4), ("torsion_min", C.c_double),
        ("grid", C.POINTER(C.POINTER(C.c_float))), ("grid_npts", C.c_int * 3), ("grid_size", C.c_double * 3),
        ("grid_shift", C.c_double * 3), ("grid_cell", C.c_double * 3),
        ("coul_grid", C.POINTER(C.c_float)), ("coul_npts", C.c_int * 3), ("coul_size", C.c_double * 3),
        ("coul_shift", C.c_double * 3), ("coul_cell", C.c_double * 3),
        ("chain_scheme", C.c_int), ("ntors", C.c_int),
        ("triclinic", C.c_int), ("hm", C.c_double * 9), ("hinv", C.c_double * 9),
        ("grid_tri", C.c_int), ("grid_ucm", C.c_double * 9), ("grid_ucinv", C.c_double * 9),
    ]


class MCParams(C.Structure):
    _fields_ = [("cum", C.c_double * 6), ("max_translation", C.c_double),
                ("max_rotation", C.c_double), ("fugacity_beta_v", C.c_double),
                ("ntrial_first", C.c_int), ("ntrial", C.c_int),
                ("seed", C.c_uint64), ("system", C.c_uint32)]


class MCState(C.Structure):
    _fields_ = [("u", C.c_double * 6), ("attempts", C.c_longlong * 6),
                ("accepted", C.c_longlong * 6), ("moves", C.c_longlong),
                ("widom_sum", C.c_double), ("widom_n", C.c_double), ("u_intra", C.c_double)]


_RNG_FN = C.CFUNCTYPE(C.c_double, C.c_void_p, C.c_int)
_lib = None


def build() -> None:
    """Compile the oracle (gcc) if the library is missing or stale."""
    src = [os.path.join(HERE, f) for f in ("oracle.c", "oracle.h")]
    if os.path.exists(LIB_PATH) and all(os.path.getmtime(LIB_PATH) >= os.path.getmtime(s) for s in src):
        return
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.or_lj.restype = C.c_double
        L.or_real_ewald.restype = C.c_double
        L.or_move_delta.restype = C.c_int
        L.or_mt_uniform.restype = C.c_double
        L.or_philox_uniform.restype = C.c_double
        L.or_philox_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32]
        L.or_grid_interpolate.restype = C.c_double
        L.or_grid_interpolate_cell.restype = C.c_double
        L.or_rng_mt.restype = C.c_double
        L.or_intra_energy.restype = C.c_double
        _lib = L
    return _lib


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class Oracle:
    """A system loaded into the C oracle.

    Arrays are kept alive on the Python side; the C struct points into them.
    `from_system` builds it from a raspa2_b200.systems.System; `from_arrays`
    from explicit arrays (for example the reference's own dump)."""

    def __init__(self, box, rc, beta, eps, sig2, shift, fw_xyz, fw_type, fw_q,
                 mol_type, mol_q, mol_ref, start_bead, ewald=False, alpha=0.0,
                 kidx=None, coulomb=None, overlap=1e7, maxmol=4096, rc_cc=None, cell_matrix=None):
        from raspa2_b200 import units
        self._keep = []

        def keep(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        s = OrSys()
        s.box[:] = [float(x) for x in box]
        if cell_matrix is not None:
            # triclinic box: the cell vectors as the matrix's columns
            h = np.asarray(cell_matrix, float)
            s.triclinic = 1
            s.hm[:] = [float(x) for x in h.reshape(-1)]
            s.hinv[:] = [float(x) for x in np.linalg.inv(h).reshape(-1)]
        s.rc2_vdw = rc * rc
        s.rc2_cc = (rc_cc if rc_cc is not None else rc) ** 2
        s.overlap = overlap
        s.coulomb = units.COULOMBIC_CONVERSION_FACTOR if coulomb is None else coulomb
        s.beta = beta
        self.eps = keep(eps, np.float64)
        s.ntypes = self.eps.shape[0]
        s.eps = _ptr(self.eps)
        self.sig2 = keep(sig2, np.float64); s.sig2 = _ptr(self.sig2)
        self.shift = keep(shift, np.float64); s.shift = _ptr(self.shift)
        self.fw_xyz = keep(fw_xyz, np.float64); s.fw_xyz = _ptr(self.fw_xyz)
        s.nfw = self.fw_xyz.shape[0]
        self.fw_type = keep(fw_type, np.int32); s.fw_type = _ptr(self.fw_type, _ip)
        self.fw_q = keep(fw_q, np.float64); s.fw_q = _ptr(self.fw_q)
        self.mol_type = keep(mol_type, np.int32); s.mol_type = _ptr(self.mol_type, _ip)
        s.natom = len(self.mol_type)
        self.mol_q = keep(mol_q, np.float64); s.mol_q = _ptr(self.mol_q)
        self.mol_ref = keep(mol_ref, np.float64); s.mol_ref = _ptr(self.mol_ref)
        s.start_bead = start_bead
        s.maxmol = maxmol
        self.ads = keep(np.zeros((maxmol, s.natom, 3)), np.float64)
        s.ads_xyz = _ptr(self.ads)
        s.nmol = 0
        s.ewald = 1 if ewald else 0
        s.alpha = alpha
        if ewald:
            self.kidx = keep(kidx, np.int32)
            s.nk = self.kidx.shape[0]
            s.kidx = _ptr(self.kidx, _ip)
            self.kfactor = keep(np.zeros(s.nk), np.float64); s.kfactor = _ptr(self.kfactor)
            self.sk_fw = keep(np.zeros((s.nk, 2)), np.float64); s.sk_fw = _ptr(self.sk_fw)
            self.sk_ads = keep(np.zeros((s.nk, 2)), np.float64); s.sk_ads = _ptr(self.sk_ads)
        self.s = s
        lib().or_ewald_setup(C.byref(self.s))

    @classmethod
    def from_system(cls, sysm, maxmol=4096):
        from raspa2_b200 import systems, units
        eps, sig2, shift = sysm.lj_tables()
        pos, t, q = sysm.framework()
        kidx = systems.kvector_indices(sysm.kmax) if sysm.ewald else None
        o = cls(sysm.box, sysm.cutoff, units.beta(sysm.temperature), eps, sig2, shift,
                pos, t, q, sysm.molecule_types(), sysm.molecule.charges(),
                sysm.molecule.positions, sysm.molecule.starting_bead,
                ewald=sysm.ewald, alpha=sysm.alpha, kidx=kidx, maxmol=maxmol,
                cell_matrix=sysm.box_matrix if sysm.triclinic else None)
        if sysm.triclinic:
            # grid lookups wrap into the triclinic unit cell
            u = sysm.unit_cell_matrix
            o.s.grid_tri = 1
            o.s.grid_ucm[:] = [float(x) for x in u.reshape(-1)]
            o.s.grid_ucinv[:] = [float(x) for x in np.linalg.inv(u).reshape(-1)]
        mol = sysm.molecule
        if not mol.rigid:
            s = o.s
            s.flexible = 1
            s.bond = mol.bond
            s.bend_k = mol.bend_k * units.KELVIN_TO_ENERGY
            s.bend_theta0 = np.deg2rad(mol.bend_theta0)
            s.bend_sigma = 1.0 / np.sqrt(s.beta * s.bend_k)
            s.torsion[:] = [x * units.KELVIN_TO_ENERGY for x in mol.torsion]
            phi = np.linspace(-np.pi, np.pi, 20001)
            c = np.cos(phi)
            e = (s.torsion[0] + s.torsion[1] * (1 + c) + s.torsion[2] * (1 - (2 * c * c - 1))
                 + s.torsion[3] * (1 + c * (4 * c * c - 3)))
            s.torsion_min = e.min() - 1e-6 * (e.max() - e.min()) - 1e-12
            s.chain_scheme = sysm.chain_scheme
            s.ntors = sysm.torsion_trials
        return o

    def intra_energy(self):
        return lib().or_intra_energy(C.byref(self.s))

    def set_coulomb_grid(self, grid, npts=None, size=None, shift=None, cell=None):
        """grid: plane-major Coulomb grid of a unit probe charge; None removes it."""
        if grid is None:
            self.s.coul_grid = None
            self._coul = None
            return
        self._coul = np.ascontiguousarray(grid, np.float32)
        self.s.coul_grid = self._coul.ctypes.data_as(C.POINTER(C.c_float))
        self.s.coul_npts[:] = [int(x) for x in npts]
        self.s.coul_size[:] = [float(x) for x in size]
        self.s.coul_shift[:] = [float(x) for x in shift]
        self.s.coul_cell[:] = [float(x) for x in cell]

    def grid_derivatives_real(self, p):
        out = np.zeros(9)
        lib().or_grid_derivatives_real(C.byref(self.s), _ptr(np.ascontiguousarray(p, float)), _ptr(out))
        return out

    def grid_build_coulomb(self, npts, size, shift):
        npts = np.asarray(npts, np.int32)
        g = np.zeros((8, npts[0] + 1, npts[1] + 1, npts[2] + 1), np.float32)
        lib().or_grid_build_coulomb(C.byref(self.s), _ptr(npts, _ip), _ptr(np.asarray(size, float)),
                                    _ptr(np.asarray(shift, float)), g.ctypes.data_as(C.POINTER(C.c_float)))
        return g

    def set_grids(self, grids, npts, size, shift, cell):
        """grids: {pseudo-atom type: plane-major grid (8, nx+1, ny+1, nz+1)}
        whose lookups replace that type's framework VDW pair sums; None
        switches them off."""
        if grids is None:
            self.s.grid = None
            self._grids = None
            return
        keepg = {t: np.ascontiguousarray(g, np.float32) for t, g in grids.items()}
        tab = (C.POINTER(C.c_float) * self.s.ntypes)()
        for t, g in keepg.items():
            tab[t] = g.ctypes.data_as(C.POINTER(C.c_float))
        self._grids = (keepg, tab)
        self.s.grid = C.cast(tab, C.POINTER(C.POINTER(C.c_float)))
        self.s.grid_npts[:] = [int(x) for x in npts]
        self.s.grid_size[:] = [float(x) for x in size]
        self.s.grid_shift[:] = [float(x) for x in shift]
        self.s.grid_cell[:] = [float(x) for x in cell]

    # ---- state -------------------------------------------------------------
    @property
    def nmol(self):
        return self.s.nmol

    def set_molecules(self, xyz):
        xyz = np.asarray(xyz, float).reshape(-1, self.s.natom, 3)
        self.ads[: len(xyz)] = xyz
        self.s.nmol = len(xyz)
        lib().or_recompute_sk_ads(C.byref(self.s))

    def molecules(self):
        return self.ads[: self.s.nmol].copy()

    # ---- energies ----------------------------------------------------------
    def point(self, type_, q, p, exclude=-1):
        out = np.zeros(4)
        p = np.ascontiguousarray(p, float)
        lib().or_point_energy(C.byref(self.s), C.c_int(type_), C.c_double(q), _ptr(p),
                              C.c_int(exclude), _ptr(out))
        return out

    def point_abs(self, type_, q, p, exclude=-1):
        out = np.zeros(4)
        p = np.ascontiguousarray(p, float)
        lib().or_point_energy_abs(C.byref(self.s), C.c_int(type_), C.c_double(q), _ptr(p),
                                  C.c_int(exclude), _ptr(out))
        return out

    def ewald_delta_abs(self, old=None, new=None):
        out = np.zeros(2)
        o = np.ascontiguousarray(old if old is not None else np.zeros((0, 3)), float).reshape(-1)
        n = np.ascontiguousarray(new if new is not None else np.zeros((0, 3)), float).reshape(-1)
        na = self.s.natom
        lib().or_ewald_delta_abs(C.byref(self.s), C.c_int(len(o) // (3 * na)), _ptr(o),
                                 C.c_int(len(n) // (3 * na)), _ptr(n), _ptr(out))
        return out

    def move_delta(self, m, new_xyz):
        out = np.zeros(4)
        nx = np.ascontiguousarray(new_xyz, float)
        ov = lib().or_move_delta(C.byref(self.s), C.c_int(m), _ptr(nx), _ptr(out))
        return bool(ov), out

    def ewald_delta(self, old=None, new=None):
        out = np.zeros(3)
        sk = np.zeros((max(self.s.nk, 1), 2))
        o = np.ascontiguousarray(old if old is not None else np.zeros((0, 3)), float).reshape(-1)
        n = np.ascontiguousarray(new if new is not None else np.zeros((0, 3)), float).reshape(-1)
        na = self.s.natom
        lib().or_ewald_delta(C.byref(self.s), C.c_int(len(o) // (3 * na)), _ptr(o),
                             C.c_int(len(n) // (3 * na)), _ptr(n), _ptr(out), _ptr(sk))
        return out, sk

    def total_energy(self):
        out = np.zeros(6)
        lib().or_total_energy(C.byref(self.s), _ptr(out))
        return out

    def cbmc_insert_mt(self, seed, nf, nt):
        g = (C.c_uint64 * 313)()
        lib().or_mt_seed(g, C.c_uint64(seed))
        fn = _RNG_FN(lib().or_rng_mt)
        out = np.zeros(6)
        nx = np.zeros((self.s.natom, 3))
        lib().or_cbmc_grow(C.byref(self.s), C.c_int(nf), C.c_int(nt), fn, C.cast(g, C.c_void_p),
                           _ptr(out), _ptr(nx))
        nxt = lib().or_mt_uniform(g)
        return out, nx, nxt

    def cbmc_delete_mt(self, m, seed, nf, nt):
        g = (C.c_uint64 * 313)()
        lib().or_mt_seed(g, C.c_uint64(seed))
        fn = _RNG_FN(lib().or_rng_mt)
        out = np.zeros(6)
        lib().or_cbmc_retrace(C.byref(self.s), C.c_int(m), C.c_int(nf), C.c_int(nt), fn,
                              C.cast(g, C.c_void_p), _ptr(out))
        nxt = lib().or_mt_uniform(g)
        return out, nxt

    # ---- grids -------------------------------------------------------------
    def grid_derivatives(self, type_, p):
        out = np.zeros(8)
        p = np.ascontiguousarray(p, float)
        lib().or_grid_derivatives(C.byref(self.s), C.c_int(type_), _ptr(p), _ptr(out))
        return out

    def grid_build(self, type_, npts, size, shift):
        npts = np.ascontiguousarray(npts, np.int32)
        size = np.ascontiguousarray(size, float)
        shift = np.ascontiguousarray(shift, float)
        g = np.zeros((8, npts[0] + 1, npts[1] + 1, npts[2] + 1), np.float32)
        lib().or_grid_build(C.byref(self.s), C.c_int(type_), _ptr(npts, _ip), _ptr(size),
                            _ptr(shift), g.ctypes.data_as(C.POINTER(C.c_float)))
        return g

    # ---- MC ----------------------------------------------------------------
    def mc_run(self, params: MCParams, state: MCState, step0: int, nsteps: int):
        lib().or_mc_run(C.byref(self.s), C.byref(params), C.byref(state),
                        C.c_uint64(step0), C.c_longlong(nsteps))
        return state


def grid_interpolate(grid, npts, size, shift, cell, p, cell_matrix=None):
    """cell_matrix: the unit-cell matrix of a triclinic cell (columns a, b, c)"""
    g = np.ascontiguousarray(grid, np.float32)
    npts = np.ascontiguousarray(npts, np.int32)
    size = np.ascontiguousarray(size, float)
    shift = np.ascontiguousarray(shift, float)
    cell = np.ascontiguousarray(cell, float)
    p = np.ascontiguousarray(p, float)
    if cell_matrix is None:
        return lib().or_grid_interpolate(g.ctypes.data_as(C.POINTER(C.c_float)), _ptr(npts, _ip),
                                         _ptr(size), _ptr(shift), _ptr(cell), _ptr(p))
    m = np.ascontiguousarray(cell_matrix, float)
    mi = np.ascontiguousarray(np.linalg.inv(m), float)
    return lib().or_grid_interpolate_cell(g.ctypes.data_as(C.POINTER(C.c_float)), _ptr(npts, _ip), _ptr(size),
                                          _ptr(shift), _ptr(cell), _ptr(m), _ptr(mi), _ptr(p))


def philox_uniform(seed, system, step, slot):
    return lib().or_philox_uniform(seed, system, step, slot)


def mc_params(sysm, seed, system=0, max_translation=None, max_rotation=None):
    """MCParams for a raspa2_b200.systems.System."""
    from raspa2_b200 import units
    p = MCParams()
    p.cum[:] = list(sysm.moves.cumulative())
    p.max_translation = sysm.max_translation if max_translation is None else max_translation
    p.max_rotation = np.deg2rad(sysm.max_rotation_deg) if max_rotation is None else max_rotation
    p.fugacity_beta_v = (units.beta(sysm.temperature) * units.pressure_to_internal(sysm.pressure)
                         * sysm.volume / sysm.ideal_gas_rosenbluth)
    p.ntrial_first = sysm.trials_first_bead
    p.ntrial = sysm.trials
    p.seed = seed
    p.system = system
    return p
