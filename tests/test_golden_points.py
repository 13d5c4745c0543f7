"""The CPU oracle's per-point physics against the reference's C-oracle golden
records (KGLD), with each reference test's normalization and bound
(koral/tests/golden/{state,flux,rad,opac,implicit}_golden_tests.zig).
These pin the shared restatement that the sm_100a kernels also compile."""
import numpy as np
import pytest

from tests.kgold import DevTracker, load_kgld, run_golden


def _family_scaled(t, c, z):
    # p2u / fluxprime: rows normalized by their family's max |c| (mhd 0..9, rad 9..13)
    smhd = np.maximum(1e-300, np.abs(c[:, :9]).max(axis=1, keepdims=True))
    srad = np.maximum(1e-300, np.abs(c[:, 9:]).max(axis=1, keepdims=True))
    s = np.concatenate([np.repeat(smhd, 9, axis=1), np.repeat(srad, 4, axis=1)], axis=1)
    t.add(c / s, z / s)


def test_p2u():
    i, o = load_kgld("state/p2u")
    z = run_golden("p2u", i, 13)
    t = DevTracker()
    _family_scaled(t, o, z)
    t.check(1e-13, "p2u (family-scale normalized)")


def test_u2p_solver_hot_and_entropy():
    i, o = load_kgld("state/u2p_solver")
    z = run_golden("u2p_solver", i, 20)
    c_hot, c_ent = o[:, 0], o[:, 10]
    z_hot, z_ent = z[:, 0], z[:, 10]
    mismatch = ((c_hot == 0) != (z_hot == 0)) | ((c_ent == 0) != (z_ent == 0))
    assert int(mismatch.sum()) == 0, f"u2p outcome mismatches at {np.nonzero(mismatch)[0]}"
    th, te = DevTracker(), DevTracker()
    both = (c_hot == 0) & (z_hot == 0)
    th.add(o[both, 1:10], z[both, 1:10])
    both = (c_ent == 0) & (z_ent == 0)
    te.add(o[both, 11:20], z[both, 11:20])
    th.check(1e-8, "u2p hot prims")
    te.check(1e-8, "u2p entropy prims")


def test_check_floors_mhd():
    i, o = load_kgld("state/floors")
    z = run_golden("floors", i, 14)
    assert np.array_equal(o[:, 0], z[:, 0]), "floors return codes"
    t = DevTracker()
    t.add(o[:, 1:], z[:, 1:])
    t.check(1e-12, "check_floors_mhd")


def test_tij_and_four_vectors():
    i, o = load_kgld("state/physics_tij")
    z = run_golden("physics_tij", i, 33)
    for sl, what in [(slice(0, 16), "calc_Tij"), (slice(16, 24), "ucon/ucov"), (slice(24, 33), "bcon/bcov/bsq")]:
        t = DevTracker()
        t.add(o[:, sl], z[:, sl])
        t.check(1e-13, what)


def test_conv_vels_all_pairs():
    i, o = load_kgld("state/relele_convvels")
    z = run_golden("relele_convvels", i, 4)
    t = DevTracker()
    t.add(o, z)
    t.check(1e-13, "conv_vels")


def test_lorentz_boosts():
    i, o = load_kgld("state/relele_boost")
    z = run_golden("relele_boost", i, 24)
    t = DevTracker()
    t.add(o[:, :16], z[:, :16])
    t.check(1e-13, "Lorentz lab2ff")
    t = DevTracker()
    t.add(o[:, 16:], z[:, 16:])
    t.check(1e-13, "boost2 lab2ff/ff2lab")


def test_reconstruction():
    i, o = load_kgld("flux/recon")
    z = run_golden("recon", i, 2)
    t = DevTracker()
    t.add(o, z)
    t.check(1e-14, "avg2point")


def test_gas_wavespeeds():
    i, o = load_kgld("flux/wavespeed")
    z = run_golden("wavespeed", i, 4)
    t = DevTracker()
    t.add(o, z)
    t.check(1e-13, "gas wavespeeds l/r")


def test_flux_prime():
    i, o = load_kgld("flux/fluxprime")
    z = run_golden("fluxprime", i, 13)
    t = DevTracker()
    _family_scaled(t, o, z)
    t.check(1e-13, "f_flux_prime (family-scale normalized)")


def test_rij_and_ff_rtt():
    i, o = load_kgld("rad/rad_rij")
    z = run_golden("rad_rij", i, 21)
    s = np.maximum(1e-300, np.abs(o[:, :16]).max(axis=1, keepdims=True))
    t = DevTracker()
    t.add(o[:, :16] / s, z[:, :16] / s)
    t.check(1e-14, "calc_Rij_M1")
    t = DevTracker()
    t.add(o[:, 16:17] / s, z[:, 16:17] / s)
    t.check(1e-13, "calc_ff_Rtt")
    t = DevTracker()
    t.add(o[:, 17:], z[:, 17:])
    t.check(1e-14, "ff ucon")


def test_u2p_rad_branches():
    i, o = load_kgld("rad/rad_u2prad")
    z = run_golden("rad_u2prad", i, 6)
    assert np.array_equal(o[:, 0], z[:, 0]), "u2p_rad return codes"
    assert np.array_equal(o[:, 1], z[:, 1]), "u2p_rad corrected flags"
    s = np.maximum(np.abs(o[:, 2]), 1e-300)
    t = DevTracker()
    t.add(o[:, 2] / s, z[:, 2] / s)
    t.add(o[:, 3:], z[:, 3:])
    t.check(1e-12, "u2p_rad primitives")


def test_rad_wavespeeds():
    i, o = load_kgld("rad/rad_wavespeeds")
    z = run_golden("rad_wavespeeds", i, 8)
    t = DevTracker()
    t.add(o, z)
    t.check(1e-12, "calc_rad_wavespeeds")


def test_check_floors_rad():
    i, o = load_kgld("rad/rad_floors")
    z = run_golden("rad_floors", i, 14)
    assert np.array_equal(o[:, 0], z[:, 0])
    s = np.maximum(np.abs(o[:, 1:]), 1e-300)
    t = DevTracker()
    t.add(o[:, 1:] / s, z[:, 1:] / s)
    t.check(1e-13, "check_floors_rad")


def test_rad_state_thermo_and_opacities():
    i, o = load_kgld("rad/rad_thermo")
    z = run_golden("rad_thermo", i, 13)
    t = DevTracker()
    t.add(o[:, :6], z[:, :6])
    t.check(1e-13, "state thermo")
    s = np.maximum(1e-300, np.abs(o[:, 6:13]).max(axis=1, keepdims=True))
    t = DevTracker()
    t.add(o[:, 6:13] / s, z[:, 6:13] / s)
    t.check(1e-12, "state opacities")


def test_kappa_kappaes_chi():
    i, o = load_kgld("rad/rad_opac")
    z = run_golden("rad_opac", i, 3)
    t = DevTracker()
    t.add(o, z)
    t.check(1e-12, "calc_kappa/kappaes/chi")


def test_four_force():
    i, o = load_kgld("rad/rad_gi")
    z = run_golden("rad_gi", i, 9)
    s = z[:, 8:9]
    t = DevTracker()
    t.add(o / s, z[:, :8] / s)
    t.check(1e-12, "calc_Gi lab/ff")


def _implicit_stats(i, o, z):
    """The acceptance statistics of koral/tests/golden/implicit_golden_tests.zig:50."""
    nrec = i.shape[0]
    c_ok = o[:, 0] == 0.0
    z_ok = z[:, 0] == 0.0
    stats = dict(n=nrec, c_ok=int(c_ok.sum()), entropy_flip=0, basis=0, ok_agree=0, both_ok=0, rung_agree=0,
                 compared=0, worst=0.0)
    resid_in = []
    pairs = []
    for r in range(nrec):
        z_ent = z_ok[r] and z[r, 2] == 1
        c_ent = c_ok[r] and o[r, 2] == 1
        if c_ok[r] != z_ok[r] and (z_ent or c_ent):
            stats["entropy_flip"] += 1
            continue
        stats["basis"] += 1
        if c_ok[r] == z_ok[r]:
            stats["ok_agree"] += 1
        if c_ok[r] and z_ok[r]:
            stats["both_ok"] += 1
            if not (o[r, 1] == z[r, 1] and o[r, 2] == z[r, 2] and o[r, 3] == z[r, 3]):
                continue
            stats["rung_agree"] += 1
            for cand in (z[r, 5:18], o[r, 5:18]):
                resid_in.append(np.concatenate([i[r, :24], i[r, 24:37], cand, z[r, 1:4]]))
            pairs.append(r)
    if resid_in:
        res = run_golden("implicit_resid", np.array(resid_in), 1)[:, 0].reshape(-1, 2)
        for k, r in enumerate(pairs):
            if not (res[k, 0] < 1e-8 and res[k, 1] < 1e-8):
                continue
            stats["compared"] += 1
            cpp, zpp = o[r, 5:18], z[r, 5:18]
            vel = [2, 3, 4, 10, 11, 12]
            vmax = max(1e-14, max(max(abs(cpp[v]), abs(zpp[v])) for v in vel))
            for iv in range(13):
                sc = vmax if iv in vel else max(abs(cpp[iv]), abs(zpp[iv]), 1e-300)
                stats["worst"] = max(stats["worst"], abs(cpp[iv] - zpp[iv]) / sc)
    return stats


def test_implicit_rung_ladder():
    i, o = load_kgld("rad/rad_implicit")
    z = run_golden("rad_implicit", i, 19)
    st = _implicit_stats(i, o, z)
    print("implicit golden:", st)
    # The reference's gate (koral/tests/golden/implicit_golden_tests.zig:50-168):
    # ok-agreement with C KORAL >= 97% (307/315 here). The flips are stiff
    # records at the edge of convergence, decided by last-bit rounding of C's
    # glibc transcendentals against the fdlibm ones the Zig path uses.
    assert st["ok_agree"] * 100 >= st["basis"] * 97, st
    assert st["entropy_flip"] <= 30, st
    assert st["rung_agree"] * 10 >= st["both_ok"] * 9, st
    assert st["compared"] >= 40, st
    assert st["worst"] <= 1e-6, st


def test_metric_points():
    i, o = load_kgld("metric/metric_points")
    z = run_golden("metric_points", i, 101)
    mks2 = i[:, 0] == 10
    t = DevTracker()
    t.add(o[:, :16], z[:, :16])
    t.check(1e-13, "gcov")
    for sl, b_exact, b_mks2, what in [(slice(16, 32), 1e-13, 1e-8, "gcon"), (slice(32, 33), 1e-13, 1e-8, "gdet"),
                                      (slice(33, 36), 1e-12, 1e-8, "dlgdet"), (slice(36, 100), 1e-12, 1e-8, "kris")]:
        t = DevTracker()
        t.add(o[~mks2, sl], z[~mks2, sl])
        t.check(b_exact, what + " bl/ks/mink")
        t = DevTracker()
        t.add(o[mks2, sl], z[mks2, sl])
        t.check(b_mks2, what + " mks2")
    t = DevTracker()
    t.add(o[:, 100], z[:, 100])
    t.check(1e-13, "gttpert")


def test_coco_and_jacobians():
    i, o = load_kgld("metric/coco_dxdx")
    z = run_golden("coco_dxdx", i, 20)
    err = np.abs(o - z) / np.maximum(1.0, np.maximum(np.abs(o), np.abs(z)))
    assert np.all(err <= 1e-12), float(np.nanmax(err))


def test_corrected_christoffels_on_puffy_grid():
    i, o = load_kgld("metric/krzysie_grid")
    z = run_golden("krzysie_grid", i, 66)
    err = np.abs(o[:, :2] - z[:, :2]) / np.maximum(1.0, np.abs(o[:, :2]))
    assert np.all(err <= 1e-14)
    t = DevTracker()
    t.add(o[:, 2:], z[:, 2:])
    t.check(1e-8, "kris-corrected mks2")


def test_trans_pall_coco():
    """koral/tests/golden/state_golden_tests.zig:94: MKS2 <-> KS and MKS2 <-> BL
    primitive transforms, DevTracker bound 1e-10."""
    i, o = load_kgld("state/frames_transpall")
    z = run_golden("frames_transpall", i, 13)
    t = DevTracker()
    t.add(o, z)
    t.check(1e-10, "trans_pall_coco")


def _face_shape(nx, ny, nz, ng, dim):
    sx, sy, sz = (n + 2 * ng if n > 1 else 1 for n in (nx, ny, nz))
    return (sz + (dim == 2), sy + (dim == 1), sx + (dim == 0))


def test_flux_ct():
    """koral/tests/golden/step_golden_tests.zig:299-333: Minkowski periodic
    32x32, the records' B rows of flbx/flby set, ct.fluxCt, bound 1e-15."""
    from tests.orcsim import _bind

    lib = _bind()
    i, o = load_kgld("flux/ct")
    nx, ny, nz, ng = 32, 32, 1, 3
    fb = [np.zeros(_face_shape(nx, ny, nz, ng, d) + (3,)) for d in range(2)]
    dims, ix, iy = i[:, 0].astype(int), i[:, 1].astype(int) + ng, i[:, 2].astype(int) + ng
    for d in range(2):
        m = dims == d
        fb[d][0, iy[m], ix[m], :] = i[m, 3:6]
    lib.orc_flux_ct(nx, ny, nz, ng, fb[0].ctypes.data, fb[1].ctypes.data, None)
    got = np.array([fb[d][0, y, x, :] for d, x, y in zip(dims, ix, iy)])
    t = DevTracker()
    t.add(got, o)
    t.check(1e-15, "flux_ct")


def test_b_from_a():
    """koral/tests/golden/step_golden_tests.zig:340-372: Minkowski periodic
    32x32, A from the records, set_bc (periodic images in the ghosts),
    calc_BfromA with overwrite, bound 1e-14."""
    from tests.orcsim import _bind

    lib = _bind()
    i, o = load_kgld("flux/bfroma")
    nx, ny, nz, ng = 32, 32, 1, 3
    sx, sy = nx + 2 * ng, ny + 2 * ng
    dom = np.zeros((ny, nx, 3))
    dom[i[:, 1].astype(int), i[:, 0].astype(int)] = i[:, 2:5]
    a = np.zeros((1, sy, sx, 3))
    a[0] = dom[np.arange(-ng, ny + ng) % ny][:, np.arange(-ng, nx + ng) % nx]
    b = np.zeros_like(a)
    ext = np.array([0.0, 2 * np.pi, 0.0, 2 * np.pi, 0.0, 1.0])
    lib.orc_b_from_a(nx, ny, nz, ng, ext.ctypes.data, a.ctypes.data, b.ctypes.data)
    got = b[0, i[:, 1].astype(int) + ng, i[:, 0].astype(int) + ng]
    t = DevTracker()
    t.add(got, o)
    t.check(1e-14, "calc_BfromA")
