"""The CPU oracle against the reference's Zig self-goldens
(tests/selfgolden/puffy_{fast,full}.kslf, written by
koral/testing/selfscenarios.zig:92 `run` through tools/gen_self_golden.zig).

The gate is the reference's own: bit identity of every per-step scalar, of
u and p at both snapshots (ghosts included) and of the flag maps
(koral/tests/selfgolden_tests.zig:27-34, `selfgolden.Cmp.check`). It holds
because the shared transcendental library computes exp, log1p, cbrt, sin,
cos, tan, atan and atanh with the fdlibm algorithms that Zig's std.math and
compiler-rt use, and pow with Zig's std.math.pow scheme
(include/koral/kmath.h).
"""
import numpy as np
import pytest

from tests.kgold import GOLDEN
from tests.orcsim import OracleSim, puffy_grid, puffy_options

FIELDS = ["rho", "uu", "vx", "vy", "vz", "entr", "b1", "b2", "b3", "ee", "fx", "fy", "fz"]
# koral/testing/selfgolden.zig:52 Scalars
SCALARS = ["t", "dt", "own_dt", "tstepdenmax", "tstepdenmin", "n_radimp_failures", "n_radimp_iters"]


def scalar_row(sim):
    c = sim.counters()
    return [float(c[k]) for k in SCALARS]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def field_scale_dev(a, b):
    return np.abs(a - b).max(axis=0) / np.maximum(np.abs(b).max(axis=0), 1e-300)


@pytest.mark.parametrize("name", ["puffy_fast", "puffy_full"])
def test_oracle_steps_reproduce_zig_selfgolden_bit_for_bit(name):
    """From the post-init snapshot the oracle takes the sim's own CFL steps
    (selfscenarios.zig:92: initTimestepGuess, then step(null) per record)."""
    z = np.load(f"{GOLDEN}/{name}_kslf.npz")
    sim = OracleSim(puffy_grid(int(z["nx"]), int(z["ny"])), puffy_options())
    sc = z["scalars"]
    sim.set_state(z["p"][0], z["u"][0], z["flags"][0])
    sim.lib.orc_sim_init_timestep_guess(sim.h)
    assert np.array_equal(bits(scalar_row(sim))[3:5], bits(sc[0])[3:5])  # tstepdenmax/min of the guess
    for k in range(1, sc.shape[0]):
        sim.step()
        row = scalar_row(sim)
        assert np.array_equal(bits(row), bits(sc[k])), (k, dict(zip(SCALARS, row)), dict(zip(SCALARS, sc[k])))
    assert np.array_equal(sim.flags(), z["flags"][1])
    p = sim.prims()
    u = sim.cons()
    pz = z["p"][1].reshape(-1, 13)
    uz = z["u"][1].reshape(-1, 13)
    dp = dict(zip(FIELDS, field_scale_dev(p, pz).tolist()))
    du = dict(zip(FIELDS, field_scale_dev(u, uz).tolist()))
    assert np.array_equal(bits(p), bits(pz)), dp
    assert np.array_equal(bits(u), bits(uz)), du


@pytest.mark.parametrize("name", ["puffy_fast", "puffy_full"])
def test_oracle_init_reproduces_zig_postinit_snapshot_bit_for_bit(name):
    """The PUFFY init sequence (puffy.zig:873 initAll: limotorus prepinit,
    set_bc, B from A, set_bc, beta normalization) against the self-golden's
    snapshot 0, ghosts included."""
    z = np.load(f"{GOLDEN}/{name}_kslf.npz")
    sim = OracleSim(puffy_grid(int(z["nx"]), int(z["ny"])), puffy_options())
    fac = sim.init_puffy()
    assert 0.0 < fac < 1.0
    assert np.array_equal(sim.flags(), z["flags"][0])
    p0 = z["p"][0].reshape(-1, 13)
    u0 = z["u"][0].reshape(-1, 13)
    assert np.array_equal(bits(sim.prims()), bits(p0)), dict(zip(FIELDS, field_scale_dev(sim.prims(), p0).tolist()))
    assert np.array_equal(bits(sim.cons()), bits(u0)), dict(zip(FIELDS, field_scale_dev(sim.cons(), u0).tolist()))
