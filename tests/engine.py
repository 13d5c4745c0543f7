"""Loads the engine's Python host mirror (koral-zig_b200/koralcuda.py) by path
(the package directory name is not a Python identifier)."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "koral-zig_b200")

_mod = None


def koralcuda():
    global _mod
    if _mod is None:
        spec = importlib.util.spec_from_file_location("koralcuda", os.path.join(PKG, "koralcuda.py"))
        _mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_mod)
    return _mod
