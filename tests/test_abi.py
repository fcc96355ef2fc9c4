"""CPU-side checks of the C-ABI library: it loads without a GPU and exports
every entry point include/mps_b200.h declares (no compute calls here)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mps_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from mps_b200 import _lib
    lib = _lib.load()
    names = declared_symbols("mps_b200.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_version_and_error_strings():
    from mps_b200 import _lib
    lib = _lib.load()
    assert lib.mps_version() >= 10000
    assert lib.mps_error_string(-4) == b"neighbour count exceeded max_neighbors"


def test_invalid_arguments_rejected_without_gpu():
    import ctypes as C
    from mps_b200 import _lib
    lib = _lib.load()
    assert lib.mps_step(None, 1) == -1
    assert lib.mps_session_create(None, None, 1) == -1
    assert lib.mps_session_destroy(None) == 0


def test_params_struct_matches_config():
    from mps_b200 import _lib, workloads as W
    wl = W.small_dambreak3d()
    cfg = wl.config()
    p = _lib.params_from_config(cfg, 3)
    assert p.influence_radius_lap == cfg.influence_radius_lap == 3.1 * 0.02
    assert p.cg_tolerance == 1e-9 and p.solver_type == 1
