"""The C-ABI library loads and exports every entry point include/pggc.h declares."""
import ctypes
import os
import re

from pennsylvaniagpugraphclustering_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(pggc_[A-Za-z0-9_]+)\s*\(", txt))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("pggc_leiden_part", "pggc_louvain_part", "pggc_local_move", "pggc_build_coarse_graph",
                 "pggc_coarsen_leidenR", "pggc_generate_orderings", "pggc_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH if os.path.exists(_lib.LIB_PATH) else build.build_cuda())
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert declared_symbols() == set(_lib.EXPORTED)


def test_version_string():
    assert b"sm_100a" in _lib.lib().pggc_version()
