"""Test helpers: the golden fixtures, the CPU oracle library and the
deviation trackers of the reference's golden tests
(koral/testing/golden.zig:170 DevTracker, :199 FieldDev)."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_DIR = os.path.join(ROOT, "oracle")

_oracle = None


def oracle():
    """Load (building if needed) the CPU oracle shared library."""
    global _oracle
    if _oracle is None:
        so = os.path.join(ORACLE_DIR, "liboracle.so")
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
        _oracle = ctypes.CDLL(so)
        _oracle.orc_golden.restype = ctypes.c_int
        _oracle.orc_golden.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_int]
    return _oracle


def load_kgld(rel):
    z = np.load(os.path.join(GOLDEN, rel.replace("/", "__") + ".npz"))
    nin, nout = int(z["nin"]), int(z["nout"])
    d = np.ascontiguousarray(z["data"])
    return d[:, :nin].copy(), d[:, nin:].copy()


def run_golden(name, inp, nout):
    inp = np.ascontiguousarray(inp, dtype=np.float64)
    out = np.zeros((inp.shape[0], nout), dtype=np.float64)
    rc = oracle().orc_golden(name.encode(), inp.shape[0], inp.ctypes.data, inp.shape[1], out.ctypes.data, nout)
    assert rc == 0, f"oracle harness has no case {name}"
    return out


class DevTracker:
    """max |c - z| / max(1, |c|, |z|) over a quantity class."""

    def __init__(self):
        self.max_dev = 0.0
        self.at = None

    def add(self, c, z, rec=None):
        c = np.asarray(c, dtype=np.float64)
        z = np.asarray(z, dtype=np.float64)
        dev = np.abs(c - z) / np.maximum(1.0, np.maximum(np.abs(c), np.abs(z)))
        # a NaN deviation never wins `dev > max_dev` in the reference tracker
        dev = np.where(np.isnan(dev), 0.0, dev)
        m = float(np.max(dev)) if dev.size else 0.0
        if m > self.max_dev:
            self.max_dev = m
            self.at = rec

    def check(self, bound, what):
        assert self.max_dev <= bound, f"{what}: max dev {self.max_dev:.3e} > {bound:.1e} (rec {self.at})"
        return self.max_dev
