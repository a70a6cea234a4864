"""Imports the package directory ``piko-public_b200/`` as the module ``piko_b200``.

The directory name carries a hyphen, so it cannot be imported by name; tests,
bench.py and __graft_entry__.py call :func:`load` instead.
"""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "piko-public_b200")


def load():
    mod = sys.modules.get("piko_b200")
    if mod is not None:
        return mod
    spec = importlib.util.spec_from_file_location("piko_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["piko_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
