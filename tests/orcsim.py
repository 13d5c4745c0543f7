"""ctypes wrapper of the CPU oracle's step driver (oracle/orc_sim.cpp) and of
the C-ABI option/grid/counter structs (include/koralcuda.h), shared by the
tests and bench.py's CPU baseline."""
import ctypes
import os

import numpy as np

from tests.kgold import oracle

NV = 13
NFL = 6


from tests.engine import koralcuda

_kc = koralcuda()
KcGrid, KcOptions, KcCounters, KcScalarRow = _kc.KcGrid, _kc.KcOptions, _kc.KcCounters, _kc.KcScalarRow


_sim_bound = False


def _bind():
    global _sim_bound
    lib = oracle()
    if _sim_bound:
        return lib
    vp = ctypes.c_void_p
    lib.orc_sim_create.restype = vp
    lib.orc_sim_create.argtypes = [ctypes.POINTER(KcGrid), ctypes.POINTER(KcOptions), ctypes.c_int]
    for name in ["orc_sim_destroy", "orc_sim_init_timestep_guess"]:
        getattr(lib, name).argtypes = [vp]
        getattr(lib, name).restype = None
    lib.orc_sim_ncell.argtypes = [vp]
    lib.orc_sim_ncell.restype = ctypes.c_long
    lib.orc_sim_set_threads.argtypes = [vp, ctypes.c_int]
    for name in ["orc_sim_set_prims", "orc_sim_set_cons", "orc_sim_get_prims", "orc_sim_get_cons",
                 "orc_sim_set_flags", "orc_sim_get_flags"]:
        getattr(lib, name).argtypes = [vp, vp]
        getattr(lib, name).restype = None
    lib.orc_sim_set_counters.argtypes = [vp, ctypes.POINTER(KcCounters)]
    lib.orc_sim_get_counters.argtypes = [vp, ctypes.POINTER(KcCounters)]
    for name in ["orc_sim_set_bc", "orc_sim_calc_u2p"]:
        getattr(lib, name).argtypes = [vp]
        getattr(lib, name).restype = ctypes.c_int
    lib.orc_sim_step.argtypes = [vp, ctypes.c_double]
    lib.orc_sim_step.restype = ctypes.c_int
    lib.orc_sim_phase.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    lib.orc_sim_phase.restype = ctypes.c_int
    lib.orc_sim_get_array.argtypes = [vp, ctypes.c_int, vp]
    lib.orc_sim_get_array.restype = ctypes.c_int
    lib.orc_sim_init_puffy.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong,
                                       ctypes.POINTER(ctypes.c_double)]
    lib.orc_sim_init_puffy.restype = ctypes.c_int
    lib.orc_sim_init_stage.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong,
                                       ctypes.POINTER(ctypes.c_double)]
    lib.orc_sim_init_stage.restype = ctypes.c_int
    lib.orc_sim_scalar_row.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.POINTER(KcScalarRow)]
    lib.orc_sim_scalar_row.restype = ctypes.c_int
    lib.orc_sim_kdmp_size.argtypes = [vp]
    lib.orc_sim_kdmp_size.restype = ctypes.c_long
    lib.orc_sim_kdmp_write.argtypes = [vp, ctypes.c_uint, vp, ctypes.c_long]
    lib.orc_sim_kdmp_write.restype = ctypes.c_int
    lib.orc_sim_kdmp_load.argtypes = [vp, vp, ctypes.c_long, ctypes.POINTER(_kc.KcDumpHeader)]
    lib.orc_sim_kdmp_load.restype = ctypes.c_int
    lib.orc_flux_ct.argtypes = [ctypes.c_int] * 4 + [vp] * 3
    lib.orc_flux_ct.restype = ctypes.c_int
    lib.orc_b_from_a.argtypes = [ctypes.c_int] * 4 + [vp] * 3
    lib.orc_b_from_a.restype = ctypes.c_int
    lib.orc_options_puffy.argtypes = [ctypes.POINTER(KcOptions)]
    lib.orc_grid_puffy.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(KcGrid)]
    _sim_bound = True
    return lib


def puffy_options():
    o = KcOptions()
    _bind().orc_options_puffy(ctypes.byref(o))
    return o


def puffy_grid(nx, ny, nz=1):
    g = KcGrid()
    _bind().orc_grid_puffy(nx, ny, nz, ctypes.byref(g))
    return g


class OracleSim:
    def __init__(self, grid, opt, nthreads=None):
        self.lib = _bind()
        if nthreads is None:
            nthreads = min(8, os.cpu_count() or 1)
        self.h = self.lib.orc_sim_create(ctypes.byref(grid), ctypes.byref(opt), nthreads)
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        self.grid = grid
        self.ncell = self.lib.orc_sim_ncell(self.h)

    def close(self):
        if self.h:
            self.lib.orc_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_state(self, p, u, flags=None):
        p = np.ascontiguousarray(p, dtype=np.float64).reshape(-1)
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        assert p.size == self.ncell * NV and u.size == self.ncell * NV
        self.lib.orc_sim_set_prims(self.h, p.ctypes.data)
        self.lib.orc_sim_set_cons(self.h, u.ctypes.data)
        if flags is not None:
            f = np.ascontiguousarray(flags, dtype=np.int32).reshape(-1)
            self.lib.orc_sim_set_flags(self.h, f.ctypes.data)

    def prims(self):
        out = np.empty(self.ncell * NV)
        self.lib.orc_sim_get_prims(self.h, out.ctypes.data)
        return out.reshape(self.ncell, NV)

    def cons(self):
        out = np.empty(self.ncell * NV)
        self.lib.orc_sim_get_cons(self.h, out.ctypes.data)
        return out.reshape(self.ncell, NV)

    def flags(self):
        out = np.empty(self.ncell * NFL, dtype=np.int32)
        self.lib.orc_sim_get_flags(self.h, out.ctypes.data)
        return out.reshape(self.ncell, NFL)

    def set_counters(self, **kw):
        c = KcCounters()
        self.lib.orc_sim_get_counters(self.h, ctypes.byref(c))
        for k, v in kw.items():
            setattr(c, k, v)
        self.lib.orc_sim_set_counters(self.h, ctypes.byref(c))

    def counters(self):
        c = KcCounters()
        self.lib.orc_sim_get_counters(self.h, ctypes.byref(c))
        return {k: getattr(c, k) for k, _ in KcCounters._fields_}

    def kdmp_write(self, out_idx=0):
        """serializePrimDump (koral/io/dump.zig:100) of the oracle state."""
        n = self.lib.orc_sim_kdmp_size(self.h)
        buf = (ctypes.c_uint8 * n)()
        rc = self.lib.orc_sim_kdmp_write(self.h, out_idx, buf, n)
        if rc:
            raise RuntimeError(f"oracle KDMP write failed with status {rc}")
        return bytes(buf)

    def kdmp_load(self, data):
        """loadPrimDump (koral/io/dump.zig:143); returns (status, header dict)."""
        hd = _kc.KcDumpHeader()
        rc = self.lib.orc_sim_kdmp_load(self.h, data, len(data), ctypes.byref(hd))
        return rc, {k: getattr(hd, k) for k, _ in _kc.KcDumpHeader._fields_}

    def step(self, forced_dt=float("nan")):
        rc = self.lib.orc_sim_step(self.h, forced_dt)
        if rc:
            raise RuntimeError(f"oracle step failed with status {rc}")

    def init_puffy(self, perturb=0.0, perturb_rho=0.0, seed=0):
        """The PUFFY init sequence (prepinit, set_bc, B from A, set_bc,
        beta normalization); returns the normalization factor."""
        fac = ctypes.c_double(0.0)
        rc = self.lib.orc_sim_init_puffy(self.h, perturb, perturb_rho, seed, ctypes.byref(fac))
        if rc:
            raise RuntimeError(f"oracle init failed with status {rc}")
        return fac.value

    def init_stage(self, stage, perturb=0.0, perturb_rho=0.0, seed=0):
        """One stage of the init: 0 prepinit + set_bc, 1 B from A + set_bc,
        2 beta normalization (returns the factor)."""
        fac = ctypes.c_double(0.0)
        rc = self.lib.orc_sim_init_stage(self.h, stage, perturb, perturb_rho, seed, ctypes.byref(fac))
        if rc:
            raise RuntimeError(f"oracle init stage {stage} failed with status {rc}")
        return fac.value

    def scalar_row(self, dt=0.0, r_lum=5000.0, r_scale=15.0):
        row = KcScalarRow()
        rc = self.lib.orc_sim_scalar_row(self.h, dt, r_lum, r_scale, ctypes.byref(row))
        if rc:
            raise RuntimeError(f"oracle scalar row failed with status {rc}")
        return {k: getattr(row, k) for k, _ in KcScalarRow._fields_}

    def phase(self, which, dt=0.0):
        return self.lib.orc_sim_phase(self.h, which, dt)
