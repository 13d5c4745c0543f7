"""Parity of the sm_100a engine (libkoralcuda.so, through its C ABI) with the
CPU oracle: the per-cell batch entry points on the reference's golden record
inputs, and whole RK2IMEX steps from the reference's post-init self-golden
states. The plain FP64 engine is built without FMA contraction and shares the
oracle's per-point source, so every comparison here is bit for bit."""
import os

import numpy as np
import pytest

from tests.engine import koralcuda
from tests.kgold import GOLDEN, load_kgld, run_golden
from tests.orcsim import OracleSim

pytestmark = pytest.mark.gpu


def _kc():
    kc = koralcuda()
    kc.lib()
    return kc


MODES = [0, 1, 2]  # KC_IMPLICIT_PER_CELL, KC_IMPLICIT_COMPACTING (persistent state machine), KC_IMPLICIT_SPLIT
BATCH_MODES = [0, 1, 3, 4, 5]  # the batch entry points: per-cell, persistent, sorted, rung- and iteration-compacted


@pytest.mark.parametrize("mode", BATCH_MODES)
def test_implicit_batch_bitwise_on_golden_records(mode):
    kc = _kc()
    i, _ = load_kgld("rad/rad_implicit")
    z = run_golden("rad_implicit", i, 19)
    pp, res = kc.implicit_batch(kc.puffy_options(), i[:, :23], i[:, 23], i[:, 24:37], mode=mode)
    ok = res[:, 0] == 1
    assert np.array_equal(ok, z[:, 0] == 0.0)
    assert np.array_equal(res[ok, 3], z[ok, 1].astype(int))  # whichprim
    assert np.array_equal(res[ok, 4], z[ok, 2].astype(int))  # whicheq
    assert np.array_equal(res[ok, 2], z[ok, 4].astype(int))  # iterations
    assert np.array_equal(res[:, 1], z[:, 18].astype(int))  # rung
    assert np.array_equal(pp.view(np.uint64), z[:, 5:18].copy().view(np.uint64))


def test_u2p_batch_bitwise_on_golden_records():
    kc = _kc()
    i, _ = load_kgld("state/u2p_solver")
    geom, uu, guess = i[:, :23], i[:, 23:36], i[:, 36:49]
    z = run_golden("u2p_cascade", np.concatenate([geom, uu, guess], axis=1), 16)
    pp, fl = kc.u2p_batch(kc.puffy_options(), geom, uu, guess)
    assert np.array_equal(pp.view(np.uint64), z[:, :13].copy().view(np.uint64))
    assert np.array_equal(fl, z[:, 13:16].astype(np.int32))


def _start(name, mode=0):
    kc = _kc()
    z = np.load(f"{GOLDEN}/{name}_kslf.npz")
    nx, ny = int(z["nx"]), int(z["ny"])
    grid, opt = kc.puffy_grid(nx, ny), kc.puffy_options(implicit_mode=mode)
    gpu = kc.Sim(grid, opt)
    orc = OracleSim(grid, opt)
    sc = z["scalars"][0]
    for s in (gpu,):
        s.set_prims(z["p"][0])
        s.set_cons(z["u"][0])
        s.set_flags(z["flags"][0])
        s.initTimestepGuess()
    orc.set_state(z["p"][0], z["u"][0], z["flags"][0])
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    assert gpu.counters()["tstepdenmax"] == orc.counters()["tstepdenmax"] == sc[3]
    return z, gpu, orc


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _diff_report(a, b):
    bad = np.nonzero(_bits(a) != _bits(b))
    return f"{len(bad[0])} differing entries; first at {[x[:5] for x in bad]}"


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("nsteps", [1, 3])
def test_step_bitwise_vs_oracle_puffy_fast(nsteps, mode):
    z, gpu, orc = _start("puffy_fast", mode)
    for _ in range(nsteps):
        gpu.step()
        orc.step()
    cg, co = gpu.counters(), orc.counters()
    for k in ["t", "dt", "own_dt", "tstepdenmax", "tstepdenmin"]:
        assert cg[k] == co[k], (k, cg[k], co[k])
    for k in ["n_radimp_failures", "n_radimp_iters", "n_radimp_solves", "n_guard_recoveries"]:
        assert cg[k] == co[k], (k, cg[k], co[k])
    pg, po = gpu.p, orc.prims()
    assert np.array_equal(_bits(pg), _bits(po)), _diff_report(pg, po)
    ug, uo = gpu.u, orc.cons()
    assert np.array_equal(_bits(ug), _bits(uo)), _diff_report(ug, uo)
    assert np.array_equal(gpu.flags, orc.flags())


def _pair(grid, opt):
    kc = _kc()
    orc_opt = kc.puffy_options()
    return kc.Sim(grid, opt), OracleSim(grid, orc_opt)


def _assert_same_state(gpu, orc):
    pg, po = gpu.p, orc.prims()
    assert np.array_equal(_bits(pg), _bits(po)), _diff_report(pg, po)
    ug, uo = gpu.u, orc.cons()
    assert np.array_equal(_bits(ug), _bits(uo)), _diff_report(ug, uo)
    assert np.array_equal(gpu.flags, orc.flags())


def test_init_bitwise_vs_oracle_puffy_fast():
    kc = _kc()
    grid, opt = kc.puffy_grid(32, 30), kc.puffy_options()
    gpu, orc = _pair(grid, opt)
    fg = gpu.initPuffy()
    fo = orc.init_puffy()
    assert fg == fo
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    assert gpu.counters()["tstepdenmax"] == orc.counters()["tstepdenmax"]
    _assert_same_state(gpu, orc)


@pytest.mark.parametrize("mode", MODES)
def test_init_perturbed_3d_then_steps_bitwise(mode):
    """The bench's workload shape in small: a 3D wedge with periodic phi, the
    seeded 1e-3 u_int / rho perturbations, then CFL steps."""
    kc = _kc()
    grid, opt = kc.puffy_grid(24, 20, 8), kc.puffy_options(implicit_mode=mode)
    gpu, orc = _pair(grid, opt)
    fg = gpu.initPuffy(1e-3, 1e-3, 12345)
    fo = orc.init_puffy(1e-3, 1e-3, 12345)
    assert fg == fo
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    _assert_same_state(gpu, orc)
    for _ in range(2):
        gpu.step()
        orc.step()
    cg, co = gpu.counters(), orc.counters()
    for k in ["t", "dt", "tstepdenmax", "tstepdenmin", "n_radimp_failures", "n_radimp_iters"]:
        assert cg[k] == co[k], (k, cg[k], co[k])
    _assert_same_state(gpu, orc)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["puffy64", "puffy3d"])
def test_forced_dt_steps_bitwise_from_c_state(name, mode):
    """C KORAL's post-init state of the forced-dt step goldens (64x60, and the
    32x30x4 wedge), stepped with C's dt sequence on both sides."""
    from tests.test_oracle_kstp import load_domain

    kc = _kc()
    z = np.load(f"{GOLDEN}/{name}_kstp.npz")
    grid, opt = kc.puffy_grid(int(z["nx"]), int(z["ny"]), int(z["nz"])), kc.puffy_options(implicit_mode=mode)
    gpu, orc = _pair(grid, opt)
    load_domain(orc, grid, z, 0)
    gpu.set_prims(orc.prims())
    gpu.set_cons(orc.cons())
    gpu.set_flags(orc.flags())
    gpu.setBc()
    assert orc.lib.orc_sim_set_bc(orc.h) == 0
    gpu.initTimestepGuess()
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    for k in range(1, z["t"].shape[0]):
        gpu.step(float(z["dt"][k]))
        orc.step(float(z["dt"][k]))
    assert gpu.counters()["n_radimp_iters"] == orc.counters()["n_radimp_iters"]
    _assert_same_state(gpu, orc)


def _scalars_equal(rg, ro):
    for k in rg:
        a, b = rg[k], ro[k]
        if isinstance(a, float):
            assert np.float64(a).view(np.uint64) == np.float64(b).view(np.uint64), (k, a, b)
        else:
            assert a == b, (k, a, b)


def test_scalar_row_bitwise_vs_oracle_2d_after_steps():
    """dump.scalarRow on the engine (ordered device folds) against the oracle's
    serial loops, from the puffy_fast snapshot after 3 CFL steps."""
    z, gpu, orc = _start("puffy_fast")
    for _ in range(3):
        gpu.step()
        orc.step()
    _scalars_equal(gpu.scalars(0.5, 5000.0, 15.0), orc.scalar_row(0.5, 5000.0, 15.0))
    # a shell inside the domain for the luminosity (r_lum = 50)
    _scalars_equal(gpu.scalars(0.0, 50.0, 30.0), orc.scalar_row(0.0, 50.0, 30.0))


def test_scalar_row_bitwise_vs_oracle_3d():
    kc = _kc()
    grid, opt = kc.puffy_grid(24, 20, 8), kc.puffy_options()
    gpu, orc = _pair(grid, opt)
    gpu.initPuffy(1e-3, 1e-3, 7)
    orc.init_puffy(1e-3, 1e-3, 7)
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    gpu.step()
    orc.step()
    _scalars_equal(gpu.scalars(0.0, 40.0, 15.0), orc.scalar_row(0.0, 40.0, 15.0))


@pytest.mark.parametrize("mode", MODES)
def test_graph_replay_matches_oracle(mode):
    """The step as a captured CUDA graph (kc_set_graph): the first step runs
    eagerly, the second is captured, the rest replay it with each step's own dt
    (CFL and forced); every state matches the oracle bit for bit, and a change
    of form mid-run re-captures."""
    kc = _kc()
    grid, opt = kc.puffy_grid(24, 20, 8), kc.puffy_options(implicit_mode=mode)
    gpu, orc = _pair(grid, opt)
    assert gpu.initPuffy(1e-3, 1e-3, 777) == orc.init_puffy(1e-3, 1e-3, 777)
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    gpu.set_graph(True)
    n0 = gpu.launch_count()
    for k in range(5):
        forced = None if k != 3 else 0.8 * orc.counters()["dt"]
        gpu.step(forced)
        orc.step(float("nan") if forced is None else forced)
        _assert_same_state(gpu, orc)
    per_step = (gpu.launch_count() - n0) / 5
    assert per_step == int(per_step) and per_step > 50
    cg, co = gpu.counters(), orc.counters()
    for k in ["t", "dt", "tstepdenmax", "tstepdenmin", "n_radimp_failures", "n_radimp_iters", "n_radimp_solves"]:
        assert cg[k] == co[k], (k, cg[k], co[k])
    other = 1 if mode != 1 else 0
    assert kc.lib().kc_set_implicit_mode(gpu._h, other) == 0
    for _ in range(3):
        gpu.step()
        orc.step()
        _assert_same_state(gpu, orc)


def test_autotune_restores_state_and_keeps_bits():
    """kc_autotune times candidates from a snapshot, restores the state and the
    counters, and leaves a configuration whose steps are bit-identical to the
    default one's."""
    kc = _kc()
    grid = kc.puffy_grid(48, 40, 8)
    a, b = kc.Sim(grid, kc.puffy_options()), kc.Sim(grid, kc.puffy_options())
    for s in (a, b):
        s.initPuffy(1e-3, 1e-3, 99)
        s.step()
    p0, c0 = b.p, b.counters()
    r = b.autotune(1)
    assert r["implicit_mode"] in (0, 2) and r["trials"] >= 2
    assert r["tpb_implicit"] in (256, 384, 512) and r["implicit_warps"] == r["tpb_implicit"] // 32
    for k in ("tpb_flux", "tpb_u2p"):
        assert r[k] in (64, 96, 128)
    assert r["implicit_phi_fastest"] in (0, 1)
    assert np.array_equal(b.p, p0) and b.counters() == c0
    b.set_graph(True)
    for _ in range(3):
        a.step()
        b.step()
    assert np.array_equal(a.p, b.p) and np.array_equal(a.u, b.u) and np.array_equal(a.flags, b.flags)
    assert a.counters() == b.counters()


def test_production_2d_grid_ten_steps_bitwise():
    """The 2D production configuration (384x360 PUFFY grid, the engine's own
    init, 10 CFL steps in the graph form): every state and counter identical to
    the oracle's after each step."""
    kc = _kc()
    grid = kc.puffy_grid(384, 360)
    gpu = kc.Sim(grid, kc.puffy_options())
    orc = OracleSim(grid, kc.puffy_options(), nthreads=os.cpu_count() or 1)
    assert gpu.initPuffy() == orc.init_puffy()
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    _assert_same_state(gpu, orc)
    gpu.set_graph(True)
    for _ in range(10):
        gpu.step()
        orc.step()
        _assert_same_state(gpu, orc)
    cg, co = gpu.counters(), orc.counters()
    for k in ["t", "dt", "tstepdenmax", "tstepdenmin", "n_radimp_failures", "n_radimp_iters", "n_radimp_solves"]:
        assert cg[k] == co[k], (k, cg[k], co[k])


def _face_shape(nx, ny, nz, ng, dim):
    sx, sy, sz = (n + 2 * ng if n > 1 else 1 for n in (nx, ny, nz))
    return (sz + (dim == 2), sy + (dim == 1), sx + (dim == 0))


def _oracle_flux_ct(nx, ny, nz, ng, fb):
    from tests.orcsim import _bind

    out = [None if f is None else f.copy() for f in fb]
    _bind().orc_flux_ct(nx, ny, nz, ng, *[None if f is None else f.ctypes.data for f in out])
    return out


def test_flux_ct_device_on_golden_records():
    """kc_flux_ct (the step's flux-CT kernels) on the reference's flux/ct
    golden records (koral/tests/golden/step_golden_tests.zig:299): bit for
    bit with the oracle, and within the reference's 1e-15 of C's outputs."""
    kc = _kc()
    i, o = load_kgld("flux/ct")
    nx, ny, nz, ng = 32, 32, 1, 3
    fb = [np.zeros(_face_shape(nx, ny, nz, ng, d) + (3,)) for d in range(2)] + [None]
    dims, ix, iy = i[:, 0].astype(int), i[:, 1].astype(int) + ng, i[:, 2].astype(int) + ng
    for d in range(2):
        m = dims == d
        fb[d][0, iy[m], ix[m], :] = i[m, 3:6]
    g = kc.flux_ct(nx, ny, nz, ng, fb)
    z = _oracle_flux_ct(nx, ny, nz, ng, fb)
    for d in range(2):
        assert np.array_equal(_bits(g[d]), _bits(z[d]))
    got = np.array([g[d][0, y, x, :] for d, x, y in zip(dims, ix, iy)])
    assert np.max(np.abs(got - o) / np.maximum(1.0, np.maximum(np.abs(got), np.abs(o)))) <= 1e-15


@pytest.mark.parametrize("shape", [(12, 10, 6), (1, 9, 7), (8, 1, 5)])
def test_flux_ct_device_3d_bitwise(shape):
    """Random face fluxes on 3D and collapsed-dimension grids (the 0.25 and
    0.5 EMF coefficients, pinned indices): device == oracle bit for bit."""
    kc = _kc()
    nx, ny, nz = shape
    ng = 3
    rng = np.random.default_rng(sum(shape))
    fb = [rng.standard_normal(_face_shape(nx, ny, nz, ng, d) + (3,)) if n > 1 else None
          for d, n in enumerate(shape)]
    g = kc.flux_ct(nx, ny, nz, ng, fb)
    z = _oracle_flux_ct(nx, ny, nz, ng, fb)
    for d in range(3):
        if fb[d] is not None:
            assert np.array_equal(_bits(g[d]), _bits(z[d])), d


@pytest.mark.parametrize("tiles", [1, 2])
def test_face_tile_forms_bitwise(tiles):
    """The y and z face sweeps through shared-memory tiles (reconstructed faces;
    and the PPM stencil rows as well): the perturbed 3D wedge and CFL steps,
    bit for bit with the oracle, and a 2D grid (y sweep only)."""
    kc = _kc()
    for nx, ny, nz in ((24, 20, 8), (32, 30, 1)):
        grid, opt = kc.puffy_grid(nx, ny, nz), kc.puffy_options()
        gpu, orc = _pair(grid, opt)
        gpu.set_face_tiles(tiles)
        assert gpu.initPuffy(1e-3, 1e-3, 77) == orc.init_puffy(1e-3, 1e-3, 77)
        orc.lib.orc_sim_init_timestep_guess(orc.h)
        for _ in range(3):
            gpu.step()
            orc.step()
        _assert_same_state(gpu, orc)


@pytest.mark.parametrize("threads", [256, 512])
def test_implicit_block_sizes_bitwise(threads):
    """The per-cell implicit kernel's other SM-wide blocks (255 and 128
    registers; the default 384 runs in every other test): the perturbed 3D
    wedge and a 2D grid, CFL steps bit for bit with the oracle, with the step
    eager and as a graph; an unknown size is rejected."""
    kc = _kc()
    for nx, ny, nz in ((24, 20, 8), (32, 30, 1)):
        grid, opt = kc.puffy_grid(nx, ny, nz), kc.puffy_options()
        gpu, orc = _pair(grid, opt)
        gpu.set_implicit_threads(threads)
        with pytest.raises(kc.KoralError):
            gpu.set_implicit_threads(128)
        assert gpu.initPuffy(1e-3, 1e-3, 78) == orc.init_puffy(1e-3, 1e-3, 78)
        orc.lib.orc_sim_init_timestep_guess(orc.h)
        for k in range(4):
            if k == 2:
                gpu.set_graph(True)
            gpu.step()
            orc.step()
        _assert_same_state(gpu, orc)
