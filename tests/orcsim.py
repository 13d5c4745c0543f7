"""ctypes wrapper of the CPU oracle's step driver (oracle/orc_sim.cpp) and of
the C-ABI option/grid/counter structs (include/koralcuda.h), shared by the
tests and bench.py's CPU baseline."""
import ctypes
import os

import numpy as np

from tests.kgold import oracle

NV = 13
NFL = 6


class KcGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("ng", ctypes.c_int32),
                ("minx", ctypes.c_double), ("maxx", ctypes.c_double), ("miny", ctypes.c_double),
                ("maxy", ctypes.c_double), ("minz", ctypes.c_double), ("maxz", ctypes.c_double)]


def _opt_fields():
    d, i = ctypes.c_double, ctypes.c_int32
    names = [
        ("abi_version", i), ("bhspin", d), ("mksr0", d), ("mksh0", d), ("mass", d), ("gam", d), ("tsteplim", d),
        ("minmod_theta", d), ("rhofloor", d), ("uurhoratiomin", d), ("uurhoratiomax", d), ("b2rhoratiomax", d),
        ("b2uuratiomax", d), ("gammamaxhd", d), ("isentropic_b2rhofloors", i), ("b2uufloor", i), ("horizon_x1", d),
        ("gammamaxrad", d), ("eradfloor", d), ("eerhoratiomin", d), ("eerhoratiomax", d), ("eeuuratiomin", d),
        ("eeuuratiomax", d), ("bremsstrahlung", i), ("synchrotron", i), ("kleinnishina", i), ("comptonization", i),
        ("synchrotron_bridge", i), ("scattering", i), ("hfrac", d), ("hefrac", d), ("mu_gas", d), ("mu_i", d),
        ("mu_e", d), ("radimp_conv", d), ("radimp_entrconv", d), ("radimp_eps", d), ("radimp_maxiter", i),
        ("radimp_convrel", d), ("radimp_convrelerr", d), ("radimp_convrelentr", d), ("radimp_convrelentrerr", d),
        ("radimp_damping_factor", d), ("radimp_max_en_change_down", d), ("radimp_max_en_change_up", d),
        ("radimp_max_damping", d), ("radimp_max_tgas_change", d), ("radimp_max_trad_change", d),
        ("radimp_threshold", d), ("radimp_start_with_bisect", i), ("radimp_scale_jacobian", i),
        ("radimp_allow_rad_ceiling", i), ("radimp_allow_entr_in_4dprim", i), ("radimp_opdamp_maxlevels", i),
        ("radimp_opdamp_factor", d), ("radimp_lag_opac", i), ("do_fixups", i), ("do_u2prad_fixups", i),
        ("do_radimp_fixups", i), ("correct_polaraxis", i), ("nccorrectpolar", i), ("radviscosity", i),
        ("alpharadvisc", d), ("maxradviscvel", d), ("dynamo", i), ("alphadynamo", d), ("thetaangle", d),
        ("alphabeta", d), ("betasaturated", d), ("expectedhr", d), ("alphaflipssign", i), ("dampbeta", i),
        ("calchronthego", i), ("reduceorderatbh", i), ("reduceorderafterfixup", i), ("dampradwavespeednearaxis", i),
        ("bc_x", i), ("bc_y", i), ("bc_z", i), ("precision", i), ("implicit_mode", i), ("device", i)]
    return names


class KcOptions(ctypes.Structure):
    _fields_ = _opt_fields()


class KcCounters(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("dt", ctypes.c_double), ("own_dt", ctypes.c_double),
                ("tstepdenmax", ctypes.c_double), ("tstepdenmin", ctypes.c_double), ("nstep", ctypes.c_int64),
                ("n_radimp_failures", ctypes.c_int64), ("n_radimp_fail_step", ctypes.c_int64),
                ("n_radimp_iters", ctypes.c_int64), ("n_radimp_solves", ctypes.c_int64),
                ("n_guard_recoveries", ctypes.c_int64)]


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

    def step(self, forced_dt=float("nan")):
        rc = self.lib.orc_sim_step(self.h, forced_dt)
        if rc:
            raise RuntimeError(f"oracle step failed with status {rc}")

    def phase(self, which, dt=0.0):
        return self.lib.orc_sim_phase(self.h, which, dt)
