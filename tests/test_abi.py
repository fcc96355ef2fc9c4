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


def test_precision_switches_validate_without_gpu():
    """mps_set_precision rejects a null session and unknown forms; the
    drop-in's mps_dropin_set_precision accepts the two forms and rejects
    others; the CLI rejects an unknown precision argument before any GPU
    work."""
    import ctypes as C
    import subprocess
    from mps_b200 import _lib
    lib = _lib.load()
    assert lib.mps_set_precision(None, _lib.PREC_MIXED) == -1
    assert lib.mps_set_precision(None, 7) == -1
    drop = C.CDLL(os.path.join(ROOT, "mps_b200", "libmps3d.so"))
    assert drop.mps_dropin_set_precision(7) == -1
    assert drop.mps_dropin_set_precision(-1) == -1
    assert drop.mps_dropin_set_precision(_lib.PREC_MIXED) == 0
    assert drop.mps_dropin_set_precision(_lib.PREC_FP64) == 0
    exe = os.path.join(ROOT, "mps_b200", "mps_sim3d")
    r = subprocess.run([exe, "cal.txt", "double"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Unknown precision 'double'" in r.stderr
    r = subprocess.run([exe, "cal.txt", "fp64", "extra"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Usage:" in r.stderr
