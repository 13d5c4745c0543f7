"""Python host mirror of the engine's C ABI (include/koralcuda.h).

`Sim` mirrors the reference's `Sim(cfg)` surface (koral/sim.zig:93): init,
step(forced_dt), cflDt, setBc, calcU2p, initTimestepGuess, finishInit, and the
p / u / flags fields in the reference's AoS layout (koral/field.zig:1-10),
so a test written against the reference reads the same here. All compute
runs in libkoralcuda.so on the GPU; there is no CPU path — constructing a
Sim without the library or a CUDA device raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# KORALCUDA_LIB selects another build of the library (e.g. a debug build)
LIB_PATH = os.environ.get("KORALCUDA_LIB") or os.path.join(HERE, "libkoralcuda.so")
NV = 13
NFLAGS = 6

KC_OK = 0
KC_ERR_INVALID_CONFIG = 1
KC_ERR_OOM = 2
KC_BC_PERIODIC, KC_BC_COPY, KC_BC_PUFFY = 0, 1, 2
KC_PLAIN_FP64, KC_MIXED = 0, 1
KC_FP32_PPM, KC_FP32_LAXF, KC_FP32_CT, KC_FP32_FLUX = 2, 4, 8, 16
KC_IMPLICIT_PER_CELL, KC_IMPLICIT_COMPACTING, KC_IMPLICIT_SPLIT, KC_IMPLICIT_SORTED, KC_IMPLICIT_RUNGS = 0, 1, 2, 3, 4
KC_IMPLICIT_ITERS = 5
KC_NPASS = 14
KC_ERR_TOO_MANY_CELLS = 9
KC_NOALLOC_MAX_CELLS = 16384
KC_GUESS_PLAIN, KC_GUESS_MLP = 0, 1
KC_ERR_KDMP_BAD_MAGIC, KC_ERR_KDMP_BAD_VERSION, KC_ERR_KDMP_DIM_MISMATCH, KC_ERR_KDMP_TRUNCATED, KC_ERR_IO = 10, 11, 12, 13, 14
KC_KDMP_HEADER_SIZE = 44
KC_MLP_IN, KC_MLP_HIDDEN, KC_MLP_OUT, KC_MLP_NWEIGHTS = 16, 64, 4, 5548


class KcScalarRow(ctypes.Structure):
    """kc_scalar_row: one row of the diagnostics series (koral/io/dump.zig:414)."""
    _fields_ = [("t", ctypes.c_double), ("dt", ctypes.c_double), ("nstep", ctypes.c_int64),
                ("mass", ctypes.c_double), ("mdot", ctypes.c_double), ("radlum", ctypes.c_double),
                ("totallum", ctypes.c_double), ("scaleheight", ctypes.c_double), ("max_pmag_ptot", ctypes.c_double),
                ("n_hd_fixup", ctypes.c_int64), ("n_radimp_fail", ctypes.c_int64), ("n_nan", ctypes.c_int64),
                ("n_floorguard", ctypes.c_int64)]


class KcGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("ng", ctypes.c_int32),
                ("minx", ctypes.c_double), ("maxx", ctypes.c_double), ("miny", ctypes.c_double),
                ("maxy", ctypes.c_double), ("minz", ctypes.c_double), ("maxz", ctypes.c_double)]


_d, _i = ctypes.c_double, ctypes.c_int32


class KcOptions(ctypes.Structure):
    _fields_ = [
        ("abi_version", _i), ("bhspin", _d), ("mksr0", _d), ("mksh0", _d), ("mass", _d), ("gam", _d),
        ("tsteplim", _d), ("minmod_theta", _d), ("rhofloor", _d), ("uurhoratiomin", _d), ("uurhoratiomax", _d),
        ("b2rhoratiomax", _d), ("b2uuratiomax", _d), ("gammamaxhd", _d), ("isentropic_b2rhofloors", _i),
        ("b2uufloor", _i), ("horizon_x1", _d), ("gammamaxrad", _d), ("eradfloor", _d), ("eerhoratiomin", _d),
        ("eerhoratiomax", _d), ("eeuuratiomin", _d), ("eeuuratiomax", _d), ("bremsstrahlung", _i),
        ("synchrotron", _i), ("kleinnishina", _i), ("comptonization", _i), ("synchrotron_bridge", _i),
        ("scattering", _i), ("hfrac", _d), ("hefrac", _d), ("mu_gas", _d), ("mu_i", _d), ("mu_e", _d),
        ("radimp_conv", _d), ("radimp_entrconv", _d), ("radimp_eps", _d), ("radimp_maxiter", _i),
        ("radimp_convrel", _d), ("radimp_convrelerr", _d), ("radimp_convrelentr", _d),
        ("radimp_convrelentrerr", _d), ("radimp_damping_factor", _d), ("radimp_max_en_change_down", _d),
        ("radimp_max_en_change_up", _d), ("radimp_max_damping", _d), ("radimp_max_tgas_change", _d),
        ("radimp_max_trad_change", _d), ("radimp_threshold", _d), ("radimp_start_with_bisect", _i),
        ("radimp_scale_jacobian", _i), ("radimp_allow_rad_ceiling", _i), ("radimp_allow_entr_in_4dprim", _i),
        ("radimp_opdamp_maxlevels", _i), ("radimp_opdamp_factor", _d), ("radimp_lag_opac", _i),
        ("do_fixups", _i), ("do_u2prad_fixups", _i), ("do_radimp_fixups", _i), ("correct_polaraxis", _i),
        ("nccorrectpolar", _i), ("radviscosity", _i), ("alpharadvisc", _d), ("maxradviscvel", _d), ("dynamo", _i),
        ("alphadynamo", _d), ("thetaangle", _d), ("alphabeta", _d), ("betasaturated", _d), ("expectedhr", _d),
        ("alphaflipssign", _i), ("dampbeta", _i), ("calchronthego", _i), ("reduceorderatbh", _i),
        ("reduceorderafterfixup", _i), ("dampradwavespeednearaxis", _i), ("bc_x", _i), ("bc_y", _i), ("bc_z", _i),
        ("precision", _i), ("implicit_mode", _i), ("device", _i)]


class KcCounters(ctypes.Structure):
    _fields_ = [("t", _d), ("dt", _d), ("own_dt", _d), ("tstepdenmax", _d), ("tstepdenmin", _d),
                ("nstep", ctypes.c_int64), ("n_radimp_failures", ctypes.c_int64),
                ("n_radimp_fail_step", ctypes.c_int64), ("n_radimp_iters", ctypes.c_int64),
                ("n_radimp_solves", ctypes.c_int64), ("n_guard_recoveries", ctypes.c_int64)]


class KcDumpHeader(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_uint32), ("ny", ctypes.c_uint32), ("nz", ctypes.c_uint32), ("nv", ctypes.c_uint32),
                ("t", _d), ("nstep", ctypes.c_uint64), ("out_idx", ctypes.c_uint32)]


class KcTuneResult(ctypes.Structure):
    _fields_ = [("implicit_mode", ctypes.c_int32), ("tpb_implicit", ctypes.c_int32), ("tpb_flux", ctypes.c_int32),
                ("tpb_u2p", ctypes.c_int32), ("ms_per_step", _d), ("ms_per_step_entry", _d),
                ("trials", ctypes.c_int32), ("implicit_phi_fastest", ctypes.c_int32),
                ("implicit_warps", ctypes.c_int32), ("face_tiles", ctypes.c_int32)]


class KcStepInfo(ctypes.Structure):
    _fields_ = [("dt", _d), ("nan_cell", ctypes.c_int64)]


_lib = None


def lib():
    """Load libkoralcuda.so (built in-tree by `make -C koral-zig_b200`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libkoralcuda.so is not built ({LIB_PATH}); run __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    P = ctypes.POINTER
    L.kc_options_puffy.argtypes = [P(KcOptions)]
    L.kc_options_puffy.restype = None
    L.kc_grid_puffy.argtypes = [i32, i32, i32, P(KcGrid)]
    L.kc_grid_puffy.restype = None
    L.kc_create.argtypes = [P(KcGrid), P(KcOptions), P(vp)]
    L.kc_destroy.argtypes = [vp]
    L.kc_destroy.restype = None
    L.kc_last_error.argtypes = [vp]
    L.kc_last_error.restype = ctypes.c_char_p
    for n in ["kc_upload_prims", "kc_upload_cons", "kc_download_prims", "kc_download_cons", "kc_upload_flags",
              "kc_download_flags"]:
        getattr(L, n).argtypes = [vp, vp]
    L.kc_set_counters.argtypes = [vp, P(KcCounters)]
    L.kc_get_counters.argtypes = [vp, P(KcCounters)]
    for n in ["kc_finish_init", "kc_init_timestep_guess", "kc_set_bc", "kc_calc_u2p"]:
        getattr(L, n).argtypes = [vp]
    L.kc_cfl_dt.argtypes = [vp, P(dbl)]
    L.kc_step.argtypes = [vp, dbl, P(KcStepInfo)]
    L.kc_step_n.argtypes = [vp, i32, dbl]
    L.kc_set_precision.argtypes = [vp, i32]
    L.kc_set_implicit_mode.argtypes = [vp, i32]
    L.kc_set_graph.argtypes = [vp, i32]
    L.kc_set_face_tiles.argtypes = [vp, i32]
    L.kc_set_implicit_threads.argtypes = [vp, i32]
    L.kc_autotune.argtypes = [vp, i32, P(KcTuneResult)]
    L.kc_set_guess.argtypes = [vp, i32, vp, i64]
    L.kc_init_puffy.argtypes = [vp, dbl, dbl, ctypes.c_uint64, P(dbl)]
    L.kc_implicit_batch.argtypes = [P(KcOptions), i64, vp, vp, vp, vp, i32]
    L.kc_u2p_batch.argtypes = [P(KcOptions), i64, vp, vp, vp, vp]
    L.kc_implicit_batch_noalloc.argtypes = [P(KcOptions), i64, vp, vp, vp, vp, i32]
    L.kc_implicit_batch_device.argtypes = [P(KcOptions), i64, vp, vp, vp, vp, i32, vp]
    L.kc_synth_implicit_cells.argtypes = [P(KcOptions), i64, ctypes.c_uint64, vp, vp, vp]
    L.kc_scalars.argtypes = [vp, dbl, dbl, dbl, P(KcScalarRow)]
    L.kc_set_pass_timing.argtypes = [vp, i32]
    L.kc_get_pass_times.argtypes = [vp, vp, vp]
    L.kc_pass_name.argtypes = [i32]
    L.kc_pass_name.restype = ctypes.c_char_p
    L.kc_get_stream.argtypes = [vp, P(vp)]
    L.kc_get_launch_count.argtypes = [vp, P(i64)]
    L.kc_harvest_implicit.argtypes = [vp, i64]
    L.kc_set_harvest_filter.argtypes = [vp, i32]
    L.kc_get_harvest.argtypes = [vp, vp, vp, i64, P(i64)]
    L.kc_guess_fallbacks.argtypes = [vp]
    L.kc_guess_fallbacks.restype = i64
    L.kc_mlp_train.argtypes = [vp, vp, i64, i32, i32, ctypes.c_float, ctypes.c_uint64, vp, vp]
    L.kc_mlp_forward.argtypes = [vp, i64, vp, vp]
    L.kc_mlp_grad.argtypes = [vp, i64, vp, vp, vp, vp]
    L.kc_fp64_peak.argtypes = [P(dbl)]
    L.kc_kdmp_write_header.argtypes = [P(KcDumpHeader), vp]
    L.kc_kdmp_parse_header.argtypes = [vp, i64, P(KcDumpHeader)]
    L.kc_kdmp_size.argtypes = [vp]
    L.kc_kdmp_size.restype = i64
    L.kc_kdmp_write.argtypes = [vp, ctypes.c_uint32, vp, i64, P(i64)]
    L.kc_kdmp_load.argtypes = [vp, vp, i64, P(KcDumpHeader)]
    L.kc_kdmp_write_file.argtypes = [vp, ctypes.c_char_p, ctypes.c_uint32]
    L.kc_kdmp_load_file.argtypes = [vp, ctypes.c_char_p, P(KcDumpHeader)]
    L.kc_debug_phase.argtypes = [vp, ctypes.c_int, dbl]
    L.kc_debug_get_array.argtypes = [vp, ctypes.c_int, vp]
    L.kc_debug_fail_allocs.argtypes = [vp, i32]
    L.kc_flux_ct.argtypes = [i32] * 5 + [vp] * 3
    for n in ["kc_create", "kc_upload_prims", "kc_upload_cons", "kc_download_prims", "kc_download_cons",
              "kc_upload_flags", "kc_download_flags", "kc_set_counters", "kc_get_counters", "kc_finish_init",
              "kc_init_timestep_guess", "kc_set_bc", "kc_calc_u2p", "kc_cfl_dt", "kc_step", "kc_step_n",
              "kc_set_precision", "kc_set_implicit_mode", "kc_set_guess", "kc_init_puffy", "kc_implicit_batch",
              "kc_u2p_batch", "kc_debug_phase", "kc_debug_get_array", "kc_set_pass_timing", "kc_get_pass_times",
              "kc_get_stream", "kc_get_launch_count", "kc_implicit_batch_noalloc", "kc_implicit_batch_device",
              "kc_synth_implicit_cells", "kc_scalars", "kc_harvest_implicit", "kc_get_harvest", "kc_mlp_train",
              "kc_mlp_forward", "kc_mlp_grad", "kc_fp64_peak", "kc_set_graph", "kc_autotune",
              "kc_kdmp_write_header", "kc_kdmp_parse_header", "kc_kdmp_write", "kc_kdmp_load", "kc_kdmp_write_file",
              "kc_kdmp_load_file", "kc_debug_fail_allocs", "kc_flux_ct", "kc_set_face_tiles", "kc_set_implicit_threads",
              "kc_set_harvest_filter"]:
        getattr(L, n).restype = ctypes.c_int
    _lib = L
    return L


def puffy_options(**overrides):
    """Sim.Options of the PUFFY problem (koral/problems/puffy/puffy.zig:210)."""
    o = KcOptions()
    lib().kc_options_puffy(ctypes.byref(o))
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


def puffy_grid(nx, ny, nz=1):
    """The PUFFY MKS2 grid (koral/problems/puffy/puffy.zig:185 makeGridNz)."""
    g = KcGrid()
    lib().kc_grid_puffy(nx, ny, nz, ctypes.byref(g))
    return g


class KoralError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"status {status}: {msg}")
        self.status = status


class Sim:
    """One engine instance: the device-resident state of the reference's Sim."""

    def __init__(self, grid, opt):
        self._lib = lib()
        self._h = ctypes.c_void_p()
        st = self._lib.kc_create(ctypes.byref(grid), ctypes.byref(opt), ctypes.byref(self._h))
        if st != KC_OK:
            msg = self._lib.kc_last_error(self._h).decode() if self._h else "kc_create failed"
            self.close()
            raise KoralError(st, msg)
        self.grid = grid
        sx = grid.nx + (2 * grid.ng if grid.nx > 1 else 0)
        sy = grid.ny + (2 * grid.ng if grid.ny > 1 else 0)
        sz = grid.nz + (2 * grid.ng if grid.nz > 1 else 0)
        self.shape = (sz, sy, sx)
        self.ncell = sx * sy * sz

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.kc_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        self.close()

    def _check(self, st):
        if st != KC_OK:
            raise KoralError(st, self._lib.kc_last_error(self._h).decode())

    # ---- fields (koral/sim.zig:224-262) ---------------------------------------
    def set_prims(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        assert p.size == self.ncell * NV
        self._check(self._lib.kc_upload_prims(self._h, p.ctypes.data))

    def set_cons(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == self.ncell * NV
        self._check(self._lib.kc_upload_cons(self._h, u.ctypes.data))

    def set_flags(self, f):
        f = np.ascontiguousarray(f, dtype=np.int32)
        assert f.size == self.ncell * NFLAGS
        self._check(self._lib.kc_upload_flags(self._h, f.ctypes.data))

    @property
    def p(self):
        out = np.empty((self.ncell, NV))
        self._check(self._lib.kc_download_prims(self._h, out.ctypes.data))
        return out

    @property
    def u(self):
        out = np.empty((self.ncell, NV))
        self._check(self._lib.kc_download_cons(self._h, out.ctypes.data))
        return out

    @property
    def flags(self):
        out = np.empty((self.ncell, NFLAGS), dtype=np.int32)
        self._check(self._lib.kc_download_flags(self._h, out.ctypes.data))
        return out

    # ---- scalars (koral/sim.zig:237-293) --------------------------------------
    def counters(self):
        c = KcCounters()
        self._check(self._lib.kc_get_counters(self._h, ctypes.byref(c)))
        return {k: getattr(c, k) for k, _ in KcCounters._fields_}

    def set_counters(self, **kw):
        c = KcCounters()
        self._check(self._lib.kc_get_counters(self._h, ctypes.byref(c)))
        for k, v in kw.items():
            setattr(c, k, v)
        self._check(self._lib.kc_set_counters(self._h, ctypes.byref(c)))

    # ---- methods (koral/sim.zig) -----------------------------------------------
    def initTimestepGuess(self):
        self._check(self._lib.kc_init_timestep_guess(self._h))

    def finishInit(self):
        self._check(self._lib.kc_finish_init(self._h))

    def setBc(self):
        self._check(self._lib.kc_set_bc(self._h))

    def calcU2p(self):
        self._check(self._lib.kc_calc_u2p(self._h))

    def cflDt(self):
        v = ctypes.c_double()
        self._check(self._lib.kc_cfl_dt(self._h, ctypes.byref(v)))
        return v.value

    def step(self, forced_dt=None):
        info = KcStepInfo()
        dt = float("nan") if forced_dt is None else float(forced_dt)
        self._check(self._lib.kc_step(self._h, dt, ctypes.byref(info)))
        return info.dt

    def set_graph(self, on):
        """Capture the step as a CUDA graph and replay it (bit-identical)."""
        self._check(self._lib.kc_set_graph(self._h, 1 if on else 0))

    def set_implicit_threads(self, threads):
        """Threads per block of the per-cell implicit kernel: 256, 384 (default)
        or 512; one block fills an SM, so this sets its register budget (all
        sizes give the same bits)."""
        self._check(self._lib.kc_set_implicit_threads(self._h, threads))

    def set_face_tiles(self, mode):
        """The y and z face sweeps' form: 0 per face, 1 reconstructed-face tiles,
        2 stencil and reconstructed-face tiles (all bit-identical)."""
        self._check(self._lib.kc_set_face_tiles(self._h, mode))

    def autotune(self, steps=2):
        """kc_autotune: pick the implicit form and block sizes by timing steps on
        the current state (restored afterwards); returns the choice."""
        r = KcTuneResult()
        self._check(self._lib.kc_autotune(self._h, steps, ctypes.byref(r)))
        return {k: getattr(r, k) for k, _ in KcTuneResult._fields_}

    def set_implicit_mode(self, mode):
        """KC_IMPLICIT_PER_CELL, KC_IMPLICIT_COMPACTING or KC_IMPLICIT_SPLIT
        (all bit-identical; the split form allocates its list here)."""
        self._check(self._lib.kc_set_implicit_mode(self._h, mode))

    def set_precision(self, mode):
        """KC_PLAIN_FP64 or KC_MIXED (FP32 reconstruction, LAXF and flux-CT)."""
        self._check(self._lib.kc_set_precision(self._h, mode))

    def scalars(self, dt=0.0, r_lum=5000.0, r_scale=15.0):
        """dump.scalarRow (koral/io/dump.zig:383) at the current state."""
        row = KcScalarRow()
        self._check(self._lib.kc_scalars(self._h, dt, r_lum, r_scale, ctypes.byref(row)))
        return {k: getattr(row, k) for k, _ in KcScalarRow._fields_}

    # ---- pass timers (koral/sim/timers.zig) and device plumbing -----------------
    def set_pass_timing(self, on):
        self._check(self._lib.kc_set_pass_timing(self._h, 1 if on else 0))

    def pass_times(self):
        """{pass name: (milliseconds, calls)} of the steps taken while timing was on."""
        ms = np.zeros(KC_NPASS)
        calls = np.zeros(KC_NPASS, dtype=np.int64)
        self._check(self._lib.kc_get_pass_times(self._h, ms.ctypes.data, calls.ctypes.data))
        return {self._lib.kc_pass_name(i).decode(): (float(ms[i]), int(calls[i])) for i in range(KC_NPASS)}

    def stream(self):
        """The handle's cudaStream_t as an integer."""
        v = ctypes.c_void_p()
        self._check(self._lib.kc_get_stream(self._h, ctypes.byref(v)))
        return v.value or 0

    def launch_count(self):
        v = ctypes.c_int64()
        self._check(self._lib.kc_get_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def initPuffy(self, perturb=0.0, perturb_rho=0.0, seed=0):
        """puffy.initAllWith (koral/problems/puffy/puffy.zig:873) + initTimestepGuess;
        returns the beta normalization factor."""
        fac = ctypes.c_double(0.0)
        self._check(self._lib.kc_init_puffy(self._h, perturb, perturb_rho, seed, ctypes.byref(fac)))
        return fac.value

    # ---- the learned initial guess of the implicit solve -------------------------
    def set_guess(self, weights=None):
        """Install a KC_MLP_NWEIGHTS-float network (KC_GUESS_MLP), or return to
        the reference's bisection warm start (weights None)."""
        if weights is None:
            self._check(self._lib.kc_set_guess(self._h, KC_GUESS_PLAIN, None, 0))
            return
        w = np.ascontiguousarray(weights, dtype=np.float32)
        self._check(self._lib.kc_set_guess(self._h, KC_GUESS_MLP, w.ctypes.data, w.size))

    def debug_fail_allocs(self, n):
        """Test hook: the n-th next optional allocation fails (KC_ERR_OOM); 0 disarms."""
        self._check(self._lib.kc_debug_fail_allocs(self._h, int(n)))

    def harvest_implicit(self, capacity):
        """Collect (features, targets) of first-rung converged solves from the
        next implicit pass on, up to `capacity` pairs (0 stops)."""
        self._check(self._lib.kc_harvest_implicit(self._h, int(capacity)))

    def set_harvest_filter(self, mode):
        """0: harvest every first-rung converged solve; 1: only those whose
        pre-solve state fails the Newton core's first residual test."""
        self._check(self._lib.kc_set_harvest_filter(self._h, mode))

    def get_harvest(self, capacity):
        x = np.empty((capacity, KC_MLP_IN), dtype=np.float32)
        t = np.empty((capacity, KC_MLP_OUT), dtype=np.float32)
        n = ctypes.c_int64(0)
        self._check(self._lib.kc_get_harvest(self._h, x.ctypes.data, t.ctypes.data, capacity, ctypes.byref(n)))
        return x[:n.value].copy(), t[:n.value].copy()

    def guess_fallbacks(self):
        return int(self._lib.kc_guess_fallbacks(self._h))

    # ---- KDMP v2 checkpoints (koral/io/dump.zig) ---------------------------------
    def kdmp_write(self, out_idx=0):
        """serializePrimDump of the device state: the KDMP file bytes."""
        n = self._lib.kc_kdmp_size(self._h)
        buf = (ctypes.c_uint8 * n)()
        w = ctypes.c_int64(0)
        self._check(self._lib.kc_kdmp_write(self._h, out_idx, buf, n, ctypes.byref(w)))
        return bytes(buf)[:w.value]

    def kdmp_load(self, data):
        """loadPrimDump: p from the file, u = p2u(p); returns the header (the
        caller adopts t / nstep and runs finishInit, as in the reference)."""
        hd = KcDumpHeader()
        self._check(self._lib.kc_kdmp_load(self._h, data, len(data), ctypes.byref(hd)))
        return {k: getattr(hd, k) for k, _ in KcDumpHeader._fields_}

    def kdmp_write_file(self, path, out_idx=0):
        self._check(self._lib.kc_kdmp_write_file(self._h, os.fsencode(path), out_idx))

    def kdmp_load_file(self, path):
        hd = KcDumpHeader()
        self._check(self._lib.kc_kdmp_load_file(self._h, os.fsencode(path), ctypes.byref(hd)))
        return {k: getattr(hd, k) for k, _ in KcDumpHeader._fields_}

    def debug_phase(self, phase, dt=0.0):
        self._check(self._lib.kc_debug_phase(self._h, phase, dt))


def implicit_batch(opt, geom23, dt, pp, mode=KC_IMPLICIT_PER_CELL):
    """solveImplicitLab over independent cells (koral/solve/implicit.zig:927)."""
    geom23 = np.ascontiguousarray(geom23, dtype=np.float64)
    dt = np.ascontiguousarray(dt, dtype=np.float64)
    pp = np.array(pp, dtype=np.float64, order="C", copy=True)
    n = pp.shape[0]
    res = np.zeros((n, 6), dtype=np.int32)
    st = lib().kc_implicit_batch(ctypes.byref(opt), n, geom23.ctypes.data, dt.ctypes.data, pp.ctypes.data,
                                 res.ctypes.data, mode)
    if st != KC_OK:
        raise KoralError(st, "kc_implicit_batch")
    return pp, res


def flux_ct(nx, ny, nz, ng, fb, device=0):
    """ct.fluxCt (koral/sim/ct.zig:38) on face-flux B rows: fb is a list of
    three arrays (None for an inactive direction) in the FaceStore layout,
    shape (FZ, FY, FX, 3); returns rebuilt copies."""
    out = [None if f is None else np.ascontiguousarray(f, dtype=np.float64).copy() for f in fb]
    ptr = [None if f is None else f.ctypes.data for f in out]
    st = lib().kc_flux_ct(device, nx, ny, nz, ng, *ptr)
    if st != KC_OK:
        raise KoralError(st, "kc_flux_ct")
    return out


def implicit_batch_noalloc(opt, geom23, dt, pp, mode=KC_IMPLICIT_PER_CELL):
    """implicit_batch staged through the library's fixed device array (no
    allocation); at most KC_NOALLOC_MAX_CELLS cells per call."""
    geom23 = np.ascontiguousarray(geom23, dtype=np.float64)
    dt = np.ascontiguousarray(dt, dtype=np.float64)
    pp = np.array(pp, dtype=np.float64, order="C", copy=True)
    n = pp.shape[0]
    res = np.zeros((n, 6), dtype=np.int32)
    st = lib().kc_implicit_batch_noalloc(ctypes.byref(opt), n, geom23.ctypes.data, dt.ctypes.data, pp.ctypes.data,
                                         res.ctypes.data, mode)
    if st != KC_OK:
        raise KoralError(st, "kc_implicit_batch_noalloc")
    return pp, res


def synth_implicit_cells(opt, n, seed):
    """Seeded synthetic (geom23, dt, pp) cells of the implicit microbenchmark."""
    geom23 = np.empty((n, 23))
    dt = np.empty(n)
    pp = np.empty((n, NV))
    st = lib().kc_synth_implicit_cells(ctypes.byref(opt), n, seed, geom23.ctypes.data, dt.ctypes.data, pp.ctypes.data)
    if st != KC_OK:
        raise KoralError(st, "kc_synth_implicit_cells")
    return geom23, dt, pp


def implicit_batch_device(opt, n, geom23_ptr, dt_ptr, pp_ptr, res_ptr, stream=0, mode=KC_IMPLICIT_PER_CELL):
    """Launch the batch solve on device arrays (raw pointers) without waiting."""
    st = lib().kc_implicit_batch_device(ctypes.byref(opt), n, geom23_ptr, dt_ptr, pp_ptr, res_ptr, mode, stream)
    if st != KC_OK:
        raise KoralError(st, "kc_implicit_batch_device")


def u2p_batch(opt, geom23, uu, pp):
    """The per-cell u2p cascade of calcU2p (koral/sim.zig:972-994)."""
    geom23 = np.ascontiguousarray(geom23, dtype=np.float64)
    uu = np.ascontiguousarray(uu, dtype=np.float64)
    pp = np.array(pp, dtype=np.float64, order="C", copy=True)
    n = pp.shape[0]
    fl = np.zeros((n, 3), dtype=np.int32)
    st = lib().kc_u2p_batch(ctypes.byref(opt), n, geom23.ctypes.data, uu.ctypes.data, pp.ctypes.data, fl.ctypes.data)
    if st != KC_OK:
        raise KoralError(st, "kc_u2p_batch")
    return pp, fl


def _status(st, what):
    if st != KC_OK:
        raise KoralError(st, what)


def mlp_train(features, targets, steps=2000, batch=1024, lr=1e-3, seed=1):
    """Train the guess network on the GPU; returns (weights blob, loss per step)."""
    x = np.ascontiguousarray(features, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    w = np.empty(KC_MLP_NWEIGHTS, dtype=np.float32)
    loss = np.empty(max(steps, 1), dtype=np.float32)
    _status(lib().kc_mlp_train(x.ctypes.data, t.ctypes.data, x.shape[0], steps, batch, lr, seed, w.ctypes.data,
                               loss.ctypes.data), "kc_mlp_train")
    return w, loss[:steps]


def mlp_forward(weights, features_std):
    """The tensor-core forward pass on standardised features (n x 16)."""
    w = np.ascontiguousarray(weights, dtype=np.float32)
    x = np.ascontiguousarray(features_std, dtype=np.float32)
    y = np.empty((x.shape[0], KC_MLP_OUT), dtype=np.float32)
    _status(lib().kc_mlp_forward(w.ctypes.data, x.shape[0], x.ctypes.data, y.ctypes.data), "kc_mlp_forward")
    return y


def mlp_grad(weights, features_std, targets_std):
    """(loss, gradient blob) of the training kernels over all pairs."""
    w = np.ascontiguousarray(weights, dtype=np.float32)
    x = np.ascontiguousarray(features_std, dtype=np.float32)
    t = np.ascontiguousarray(targets_std, dtype=np.float32)
    g = np.empty(KC_MLP_NWEIGHTS, dtype=np.float32)
    loss = ctypes.c_float(0.0)
    _status(lib().kc_mlp_grad(w.ctypes.data, x.shape[0], x.ctypes.data, t.ctypes.data, g.ctypes.data,
                              ctypes.byref(loss)), "kc_mlp_grad")
    return float(loss.value), g


def fp64_peak():
    """Measured FP64 (DFMA) peak of the current device in TFLOP/s."""
    v = ctypes.c_double(0.0)
    _status(lib().kc_fp64_peak(ctypes.byref(v)), "kc_fp64_peak")
    return v.value


def kdmp_write_header(nx, ny, nz, nv, t, nstep, out_idx):
    """writeDumpHeader (koral/io/dump.zig:67): the 44 header bytes (host only)."""
    hd = KcDumpHeader(nx, ny, nz, nv, t, nstep, out_idx)
    buf = (ctypes.c_uint8 * KC_KDMP_HEADER_SIZE)()
    _status(lib().kc_kdmp_write_header(ctypes.byref(hd), buf), "kc_kdmp_write_header")
    return bytes(buf)


def kdmp_parse_header(data):
    """parseDumpHeader (koral/io/dump.zig:86); raises KoralError with the
    reader's status (BadMagic 10, BadVersion 11, Truncated 13)."""
    hd = KcDumpHeader()
    _status(lib().kc_kdmp_parse_header(data, len(data), ctypes.byref(hd)), "kc_kdmp_parse_header")
    return {k: getattr(hd, k) for k, _ in KcDumpHeader._fields_}
