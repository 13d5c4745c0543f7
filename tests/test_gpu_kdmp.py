"""KDMP v2 checkpoints from the device state (koral/io/dump.zig) against the
oracle's serial serializer and loader: identical file bytes for identical
states, identical p and u after a load (p verbatim, u = p2u(p) on the device),
the file entry points, and the reader's errors."""
import numpy as np
import pytest

from tests.engine import koralcuda
from tests.orcsim import NV, OracleSim

pytestmark = pytest.mark.gpu


def _domain(arr, grid, ng=3):
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    gz = ng if nz > 1 else 0
    a = arr.reshape(nz + 2 * gz, ny + 2 * ng, nx + 2 * ng, NV)
    return a[gz:gz + nz, ng:ng + ny, ng:ng + nx]


def _stepped(kc, grid):
    gpu, orc = kc.Sim(grid, kc.puffy_options()), OracleSim(grid, kc.puffy_options())
    assert gpu.initPuffy(1e-3, 1e-3, 31) == orc.init_puffy(1e-3, 1e-3, 31)
    orc.lib.orc_sim_init_timestep_guess(orc.h)
    for _ in range(2):
        gpu.step()
        orc.step()
    return gpu, orc


def test_write_bytes_match_oracle_and_load_matches_oracle(tmp_path):
    kc = koralcuda()
    grid = kc.puffy_grid(24, 20, 8)
    gpu, orc = _stepped(kc, grid)
    data = gpu.kdmp_write(5)
    assert data == orc.kdmp_write(5)
    h = kc.kdmp_parse_header(data)
    assert (h["nx"], h["ny"], h["nz"], h["nv"], h["nstep"], h["out_idx"]) == (24, 20, 8, NV, 2, 5)
    assert h["t"] == gpu.counters()["t"]
    # load into fresh sims on both sides: p verbatim, u = p2u(p), bit for bit
    g2, o2 = kc.Sim(grid, kc.puffy_options()), OracleSim(grid, kc.puffy_options())
    assert g2.kdmp_load(data) == h
    assert o2.kdmp_load(data) == (0, h)
    assert np.array_equal(_domain(g2.p, grid), _domain(gpu.p, grid))
    assert np.array_equal(_domain(g2.p, grid), _domain(o2.prims(), grid))
    assert np.array_equal(_domain(g2.u, grid), _domain(o2.cons(), grid))
    # the file entry points write the same bytes and load the same state
    path = tmp_path / "frame0005.kdmp"
    gpu.kdmp_write_file(str(path), 5)
    assert path.read_bytes() == data
    g3 = kc.Sim(grid, kc.puffy_options())
    assert g3.kdmp_load_file(str(path)) == h
    assert np.array_equal(_domain(g3.u, grid), _domain(g2.u, grid))


def test_reader_errors():
    kc = koralcuda()
    grid = kc.puffy_grid(24, 20, 8)
    gpu, _ = _stepped(kc, grid)
    data = gpu.kdmp_write(0)
    other = kc.Sim(kc.puffy_grid(24, 20, 4), kc.puffy_options())
    for bad, status in ((data[:-8], kc.KC_ERR_KDMP_TRUNCATED), (b"XDMP" + data[4:], kc.KC_ERR_KDMP_BAD_MAGIC),
                        (data[:30], kc.KC_ERR_KDMP_TRUNCATED)):
        fresh = kc.Sim(grid, kc.puffy_options())
        with pytest.raises(kc.KoralError) as e:
            fresh.kdmp_load(bad)
        assert e.value.status == status
    with pytest.raises(kc.KoralError) as e:
        other.kdmp_load(data)
    assert e.value.status == kc.KC_ERR_KDMP_DIM_MISMATCH
    fresh = kc.Sim(grid, kc.puffy_options())
    with pytest.raises(kc.KoralError) as e:
        fresh.kdmp_load_file("/nonexistent/dir/x.kdmp")
    assert e.value.status == kc.KC_ERR_IO
    # a rejected file leaves the handle usable: the good one loads and the run continues
    h = fresh.kdmp_load(data)
    fresh.set_counters(t=h["t"], nstep=h["nstep"])
    fresh.finishInit()
    fresh.step()
    assert fresh.counters()["nstep"] == h["nstep"] + 1
