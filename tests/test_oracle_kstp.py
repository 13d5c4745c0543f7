"""The CPU oracle's full RK2IMEX step against C KORAL's forced-dt step goldens
(tests/golden/step/puffy64.kstp.gz: 64x60 MKS2, and puffy3d.kstp.gz: the
32x30x4 pi/2 wedge with periodic phi), with the gates of
koral/tests/golden/puffystep_golden_tests.zig:164 checkStepGolden: C's
post-init domain state is loaded, ghosts are rebuilt by set_bc, every step is
forced to C's dt, and per step (1) the entropy / hd / rad / radimp flag maps
agree cell for cell, (2) at least 95% of the cells track C to 1e-3 of each
variable's field scale, (3) no cell deviates by more than 0.15 of the field
scale, and the first (tiny-dt) step tracks to 1e-4. The 3D case exercises the
3D corner fill, periodic-z ghosts, the z sweep and the 3D B-from-A curl."""
import numpy as np
import pytest

from tests.kgold import GOLDEN
from tests.orcsim import NFL, NV, OracleSim, puffy_grid, puffy_options

# oracle flag slots of the KSTP flag columns (entropy, hd_fixup, rad_fixup, radimp_fixup)
KSTP_FLAG_SLOTS = [0, 3, 4, 5]


def load_domain(sim, grid, z, rec):
    """Domain cells of a KSTP record into a full (ghosted) oracle state."""
    nx, ny, nz = int(z["nx"]), int(z["ny"]), int(z["nz"])
    ng = 3
    sx, sy = nx + 2 * ng, ny + 2 * ng
    sz = nz + 2 * ng if nz > 1 else 1
    ngz = ng if nz > 1 else 0
    p = np.zeros((sz, sy, sx, NV))
    u = np.zeros((sz, sy, sx, NV))
    p[ngz:ngz + nz, ng:ng + ny, ng:ng + nx] = z["p"][rec].reshape(nz, ny, nx, NV)
    u[ngz:ngz + nz, ng:ng + ny, ng:ng + nx] = z["u"][rec].reshape(nz, ny, nx, NV)
    sim.set_state(p.reshape(-1, NV), u.reshape(-1, NV), np.zeros((sx * sy * sz, NFL), dtype=np.int32))
    return (slice(ngz, ngz + nz), slice(ng, ng + ny), slice(ng, ng + nx)), (sz, sy, sx)


def bl_radius(grid, nx):
    # r_BL of the x cell centers: MKS2 r = exp(x1) + mksr0, with mksr0 = 0.1... read off the grid
    dx = (grid.maxx - grid.minx) / nx
    return np.exp(grid.minx + (np.arange(nx) + 0.5) * dx) + puffy_options().mksr0


@pytest.mark.parametrize("name", ["puffy64", "puffy3d"])
def test_oracle_step_vs_c_forced_dt(name):
    z = np.load(f"{GOLDEN}/{name}_kstp.npz")
    nx, ny, nz = int(z["nx"]), int(z["ny"]), int(z["nz"])
    grid, opt = puffy_grid(nx, ny, nz), puffy_options()
    sim = OracleSim(grid, opt)
    dom, shape = load_domain(sim, grid, z, 0)
    assert sim.lib.orc_sim_set_bc(sim.h) == 0
    sim.lib.orc_sim_init_timestep_guess(sim.h)
    ncp = opt.nccorrectpolar
    rbl = bl_radius(grid, nx)
    rows = []
    for k in range(1, z["t"].shape[0]):
        sim.step(float(z["dt"][k]))
        t = sim.counters()["t"]
        assert abs(t - z["t"][k]) <= 1e-11 * abs(z["t"][k])
        cp = z["p"][k].reshape(nz, ny, nx, NV)
        zp = sim.prims().reshape(*shape, NV)[dom]
        scale = np.maximum(np.abs(cp).max(axis=(0, 1, 2)), 1e-300)
        cf = z["flags"][k].reshape(nz, ny, nx, -1)
        zf = sim.flags().reshape(*shape, NFL)[dom][..., KSTP_FLAG_SLOTS[:cf.shape[-1]]]
        ok = np.all(cf == zf, axis=-1)
        dev = (np.abs(cp - zp) / scale).max(axis=-1)
        dev_ok = np.where(ok, dev, 0.0)
        interior = (rbl[None, None, :] >= 2.5) & (np.arange(ny)[None, :, None] > ncp) & \
            (np.arange(ny)[None, :, None] < ny - 1 - ncp)
        rows.append(dict(step=k, flags=float(ok.mean()), max=float(dev_ok.max()),
                         interior=float(np.where(interior, dev_ok, 0).max()), over=float((dev_ok > 1e-3).mean())))
    print(name, rows)
    for r in rows:
        assert r["flags"] == 1.0, r
        assert r["over"] <= 0.05, r
        assert r["max"] <= 0.15, r
    assert rows[0]["max"] <= 1e-4, rows[0]
