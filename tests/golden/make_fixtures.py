"""Convert the reference's committed golden files into the compact .npz
fixtures the tests read.

The reference (koral-zig) keeps three golden families for the step path:
  * KGLD  — per-function C-oracle records (koral/testing/golden.zig:32):
            "KGLD" u32 version, u64 nrec, u32 nin, u32 nout, f64 data[]
  * KSTP  — forced-dt full-step records of C KORAL (golden.zig:58), optionally
            gzipped: "KSTP" u32 version, u32 nx,ny,nz,nv, u64 nrec, then per
            record {t, dt, u[ncell*nv], p[ncell*nv], flags[nf*ncell]}
  * KSLF  — Zig self-goldens (koral/testing/selfgolden.zig:20), gzipped.
  * KINI  — C KORAL's PUFFY t=0 init snapshots (golden.zig:313 readKini),
            gzipped: "KINI" u32 version, i32 nx,ny,nz,gx,gy,gz,stride,nvars,
            i32 vars[nvars], f64 data[] (iz slowest, then iy, ix, vars fastest;
            ghosts included when gx/gy > 0, else a stride-sampled domain).

This script is run once where the reference tree is available; its outputs
under tests/golden/ are what the test suite (and the GPU box) reads.

    python tests/golden/make_fixtures.py /path/to/koral-zig
"""
import gzip
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

KGLD = [
    "state/p2u.kgld", "state/u2p_solver.kgld", "state/floors.kgld", "state/physics_tij.kgld",
    "state/relele_convvels.kgld", "state/relele_boost.kgld", "state/frames_transpall.kgld",
    "flux/recon.kgld", "flux/wavespeed.kgld", "flux/fluxprime.kgld", "flux/ct.kgld", "flux/bfroma.kgld",
    "rad/rad_rij.kgld", "rad/rad_u2prad.kgld", "rad/rad_wavespeeds.kgld", "rad/rad_floors.kgld",
    "rad/rad_thermo.kgld", "rad/rad_opac.kgld", "rad/rad_gi.kgld", "rad/rad_implicit.kgld",
    "metric/metric_points.kgld", "metric/coco_dxdx.kgld", "metric/krzysie_grid.kgld",
    "init/puffy_scalars.kgld",
]
KINI = ["init/puffy_t0_A.kini.gz", "init/puffy_t0_eps12.kini.gz", "init/puffy_t0_pfinal.kini.gz"]
KSLF = ["puffy_fast.kslf", "puffy_full.kslf"]
KSTP = ["step/puffy64.kstp.gz", "step/puffy3d.kstp.gz"]


def read_maybe_gz(path):
    raw = open(path, "rb").read()
    if raw[:2] == b"\x1f\x8b":
        raw = gzip.decompress(raw)
    return raw


def conv_kgld(src, dst):
    raw = open(src, "rb").read()
    assert raw[:4] == b"KGLD" and struct.unpack("<I", raw[4:8])[0] == 1
    nrec = struct.unpack("<Q", raw[8:16])[0]
    nin, nout = struct.unpack("<II", raw[16:24])
    data = np.frombuffer(raw[24:], dtype="<f8").reshape(nrec, nin + nout)
    np.savez_compressed(dst, nin=nin, nout=nout, data=data)


def conv_kslf(src, dst):
    raw = read_maybe_gz(src)
    assert raw[:4] == b"KSLF"
    version, nx, ny, nz, ng, nv = struct.unpack("<IIIIII", raw[4:28])
    (ncell,) = struct.unpack("<Q", raw[28:36])
    nflags, nsc, nfield, llen = struct.unpack("<IIII", raw[36:52])
    off = 52 + llen
    off += (8 - off % 8) % 8
    vals = np.frombuffer(raw[off:], dtype="<f8")
    nscv = nsc * 7
    scalars = vals[:nscv].reshape(nsc, 7)
    steps = vals[nscv:nscv + nfield]
    fl = vals[nscv + nfield:].reshape(nfield, -1)
    nu = ncell * nv
    u = fl[:, :nu].reshape(nfield, ncell, nv)
    p = fl[:, nu:2 * nu].reshape(nfield, ncell, nv)
    flags = fl[:, 2 * nu:].reshape(nfield, ncell, nflags).astype(np.int32)
    np.savez_compressed(dst, nx=nx, ny=ny, nz=nz, ng=ng, nv=nv, scalars=scalars, steps=steps, u=u, p=p, flags=flags,
                        label=raw[52:52 + llen].decode())


def conv_kstp(src, dst):
    raw = read_maybe_gz(src)
    assert raw[:4] == b"KSTP"
    version, nx, ny, nz, nv = struct.unpack("<IIIII", raw[4:24])
    (nrec,) = struct.unpack("<Q", raw[24:32])
    ncell = nx * ny * nz
    vals = np.frombuffer(raw[32:], dtype="<f8").reshape(nrec, -1)
    per = vals.shape[1]
    nf = (per - 2 - 2 * ncell * nv) // ncell
    nu = ncell * nv
    np.savez_compressed(dst, nx=nx, ny=ny, nz=nz, nv=nv, t=vals[:, 0], dt=vals[:, 1],
                        u=vals[:, 2:2 + nu].reshape(nrec, ncell, nv), p=vals[:, 2 + nu:2 + 2 * nu].reshape(nrec, ncell, nv),
                        flags=vals[:, 2 + 2 * nu:].reshape(nrec, ncell, nf).astype(np.int32))


def conv_kini(src, dst):
    raw = read_maybe_gz(src)
    assert raw[:4] == b"KINI" and struct.unpack("<I", raw[4:8])[0] == 1
    nx, ny, nz, gx, gy, gz, stride, nvars = struct.unpack("<8i", raw[8:40])
    vars_ = np.frombuffer(raw[40:40 + 4 * nvars], dtype="<i4").copy()
    sx = nx + 2 * gx if gx > 0 else (nx + stride - 1) // stride
    sy = ny + 2 * gy if gy > 0 else (ny + stride - 1) // stride
    data = np.frombuffer(raw[40 + 4 * nvars:], dtype="<f8").reshape(nz, sy, sx, nvars)
    np.savez_compressed(dst, nx=nx, ny=ny, nz=nz, gx=gx, gy=gy, gz=gz, stride=stride, vars=vars_, data=data)


def main(ref):
    for rel in KGLD:
        dst = os.path.join(HERE, rel.replace("/", "__").replace(".kgld", ".npz"))
        conv_kgld(os.path.join(ref, "tests/golden", rel), dst)
    for rel in KSLF:
        conv_kslf(os.path.join(ref, "tests/selfgolden", rel), os.path.join(HERE, rel.replace(".kslf", "_kslf.npz")))
    for rel in KINI:
        name = os.path.basename(rel).replace(".kini.gz", "_kini.npz")
        conv_kini(os.path.join(ref, "tests/golden", rel), os.path.join(HERE, name))
    for rel in KSTP:
        name = os.path.basename(rel).replace(".kstp.gz", "_kstp.npz")
        conv_kstp(os.path.join(ref, "tests/golden", rel), os.path.join(HERE, name))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_fixtures.py <koral-zig checkout>")
    main(sys.argv[1])
