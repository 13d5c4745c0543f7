"""The C-ABI boundary without a GPU: libkoralcuda.so loads, exports every
function include/koralcuda.h declares, and its host-only entry points (option
and grid defaults, pass names, argument validation, the no-device error path)
behave as documented. No kernel is launched here."""
import ctypes
import os
import re

import pytest

from tests.engine import ROOT, koralcuda

HEADER = os.path.join(ROOT, "include", "koralcuda.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(kc_[a-z_0-9]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    lib = koralcuda().lib()
    names = declared_functions()
    assert len(names) >= 30, names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_option_and_grid_defaults_match_puffy():
    kc = koralcuda()
    o = kc.puffy_options()
    assert o.abi_version == 1
    assert o.gam == pytest.approx(5.0 / 3.0)
    assert o.mass == 10.0 and o.bhspin == 0.0
    g = kc.puffy_grid(192, 180, 64)
    assert (g.nx, g.ny, g.nz, g.ng) == (192, 180, 64, 3)
    assert g.minx == pytest.approx(__import__("math").log(1.85 - 0.1))
    assert g.maxz == pytest.approx(__import__("math").pi / 4)


def test_pass_names_mirror_reference_timers():
    lib = koralcuda().lib()
    names = [lib.kc_pass_name(i).decode() for i in range(koralcuda().KC_NPASS)]
    assert names[0] == "step" and "implicit" in names and "fluxes" in names and "fluxct" in names
    assert lib.kc_pass_name(99) == b""


def test_null_arguments_are_rejected_not_crashed():
    kc = koralcuda()
    lib = kc.lib()
    assert lib.kc_create(None, None, None) == kc.KC_ERR_INVALID_CONFIG
    assert lib.kc_step(None, float("nan"), None) == kc.KC_ERR_INVALID_CONFIG
    assert lib.kc_get_stream(None, None) == kc.KC_ERR_INVALID_CONFIG
    assert lib.kc_set_pass_timing(None, 1) == kc.KC_ERR_INVALID_CONFIG


def test_invalid_config_is_reported_before_any_device_work():
    kc = koralcuda()
    lib = kc.lib()
    g = kc.puffy_grid(32, 30, 1)
    g.ng = 2  # PPM needs 3 ghosts
    h = ctypes.c_void_p()
    st = lib.kc_create(ctypes.byref(g), ctypes.byref(kc.puffy_options()), ctypes.byref(h))
    assert st == kc.KC_ERR_INVALID_CONFIG
    if h.value:
        lib.kc_destroy(h)


def test_create_without_a_device_fails_loudly():
    """With no CUDA device visible the engine refuses to create a handle (there
    is no CPU fallback)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    kc = koralcuda()
    with pytest.raises(kc.KoralError):
        kc.Sim(kc.puffy_grid(32, 30), kc.puffy_options())


STRUCTS = {"kc_grid": "KcGrid", "kc_options": "KcOptions", "kc_counters": "KcCounters",
           "kc_step_info": "KcStepInfo", "kc_scalar_row": "KcScalarRow", "kc_tune_result": "KcTuneResult",
           "kc_dump_header": "KcDumpHeader"}


def test_ctypes_mirror_matches_header_layouts(tmp_path):
    """Every POD struct of the header has the same size and field offsets in the
    Python mirror (a C program built here prints them from the header itself)."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    kc = koralcuda()
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "koralcuda.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in getattr(kc, pyname)._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            name, field, val = ln.split()
            got[(name, field)] = int(val)
    for cname, pyname in STRUCTS.items():
        cls = getattr(kc, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
