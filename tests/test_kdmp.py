"""KDMP v2 checkpoints (koral/io/dump.zig) on the CPU: the header codec of the
engine's C ABI (host-only entry points) against the reference's layout and its
tests (dump.zig:471 round trip, :480 bad magic / version / truncation), and the
oracle's serializer/loader round trip (koral/tests/restart_tests.zig:71: p and
u bit for bit, clock / step / frame restored; :127 shape mismatch rejected)."""
import struct

import numpy as np
import pytest

from tests.engine import koralcuda
from tests.orcsim import NV, OracleSim, puffy_grid, puffy_options


def test_header_layout_and_round_trip():
    kc = koralcuda()
    b = kc.kdmp_write_header(384, 360, 4, 13, 123.456, 98765, 42)
    assert len(b) == 44 == kc.KC_KDMP_HEADER_SIZE
    assert b == struct.pack("<4sIIIIIdQI", b"KDMP", 2, 384, 360, 4, 13, 123.456, 98765, 42)
    h = kc.kdmp_parse_header(b)
    assert h == {"nx": 384, "ny": 360, "nz": 4, "nv": 13, "t": 123.456, "nstep": 98765, "out_idx": 42}


def test_header_rejects_bad_magic_version_truncation():
    kc = koralcuda()
    b = kc.kdmp_write_header(1, 1, 1, 13, 0.0, 0, 0)
    with pytest.raises(kc.KoralError) as e:
        kc.kdmp_parse_header(b[:43])
    assert e.value.status == kc.KC_ERR_KDMP_TRUNCATED
    with pytest.raises(kc.KoralError) as e:
        kc.kdmp_parse_header(b"X" + b[1:])
    assert e.value.status == kc.KC_ERR_KDMP_BAD_MAGIC
    with pytest.raises(kc.KoralError) as e:
        kc.kdmp_parse_header(b[:4] + struct.pack("<I", 999) + b[8:])
    assert e.value.status == kc.KC_ERR_KDMP_BAD_VERSION


def _domain(arr, grid, ng=3):
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    gz = ng if nz > 1 else 0
    a = arr.reshape(nz + 2 * gz, ny + 2 * ng, nx + 2 * ng, NV)
    return a[gz:gz + nz, ng:ng + ny, ng:ng + nx]


def test_oracle_round_trip_bitwise():
    """The init state (every domain cell has u = p2u(p), as restart_tests.zig's
    initCell pattern does) reloads bit for bit in p and u."""
    grid = puffy_grid(24, 20, 4)
    src = OracleSim(grid, puffy_options())
    src.init_puffy(1e-3, 1e-3, 5)
    src.set_counters(t=12.3456789, nstep=4242)
    data = src.kdmp_write(7)
    assert len(data) == 44 + 24 * 20 * 4 * NV * 8
    body = np.frombuffer(data[44:], dtype="<f8").reshape(4, 20, 24, NV)
    assert np.array_equal(body, _domain(src.prims(), grid))
    dst = OracleSim(grid, puffy_options())
    rc, h = dst.kdmp_load(data)
    assert rc == 0
    assert h == {"nx": 24, "ny": 20, "nz": 4, "nv": NV, "t": 12.3456789, "nstep": 4242, "out_idx": 7}
    assert np.array_equal(_domain(dst.prims(), grid), _domain(src.prims(), grid))
    assert np.array_equal(_domain(dst.cons(), grid), _domain(src.cons(), grid))
    wrong = OracleSim(puffy_grid(25, 20, 4), puffy_options())
    assert wrong.kdmp_load(data)[0] == koralcuda().KC_ERR_KDMP_DIM_MISMATCH
    assert dst.kdmp_load(data[:-8])[0] == koralcuda().KC_ERR_KDMP_TRUNCATED
    for s in (src, dst, wrong):
        s.close()


def test_oracle_stepped_state_reloads_primitives():
    """After a step u is the evolved conserved state, not p2u(p); the restart
    trusts the primitives (dump.zig:139): p comes back bit for bit, u is p2u
    of it, and u differs from the evolved one by round-off only."""
    grid = puffy_grid(24, 20, 4)
    src = OracleSim(grid, puffy_options())
    src.init_puffy(1e-3, 1e-3, 5)
    src.lib.orc_sim_init_timestep_guess(src.h)
    src.step()
    data = src.kdmp_write(1)
    dst = OracleSim(grid, puffy_options())
    assert dst.kdmp_load(data)[0] == 0
    assert np.array_equal(_domain(dst.prims(), grid), _domain(src.prims(), grid))
    ud, us = _domain(dst.cons(), grid), _domain(src.cons(), grid)
    scale = np.abs(us).reshape(-1, NV).max(0)
    assert np.all(np.abs(ud - us).reshape(-1, NV).max(0) <= 1e-9 * np.maximum(scale, 1e-300))
    for s in (src, dst):
        s.close()
