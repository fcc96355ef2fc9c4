"""CPU checks of the drop-in's host-side functions against the reference
built from source (oracle/_ref, the reference's own io.c and sim_config.c):
the deck loaders (the drop-in's C ones and the Python package's
mps_b200.config.load_deck) fill SimConfig byte for byte as the reference's
do, and the CSV and legacy-VTK writers produce byte-identical files, in 3-D
and 2-D.
No GPU is touched: these functions only read and write host memory."""
import ctypes as C
import os

import numpy as np
import pytest

from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _libs(dim):
    ref = os.path.join(ROOT, "oracle", "_ref", f"libref{dim}d.so")
    if not os.path.exists(ref):
        pytest.skip("the reference build (oracle/_ref) is absent")
    libs = (C.CDLL(os.path.join(ROOT, "mps_b200", f"libmps{dim}d.so")), C.CDLL(ref))
    SC = T.sim_config_type(dim)
    for lib in libs:
        lib.config_set_defaults.argtypes = [C.POINTER(SC)]
        lib.config_load_cal.argtypes = [C.c_char_p, C.POINTER(SC)]
        lib.config_load_params.argtypes = [C.c_char_p, C.POINTER(SC)]
        lib.output_csv.argtypes = [C.POINTER(T.ParticleSystem), C.c_int, C.c_char_p]
        lib.output_vtk.argtypes = [C.POINTER(T.ParticleSystem), C.c_int, C.c_char_p]
    return libs


def _case(dim):
    if dim == 3:
        return W.small_dambreak3d(l0=0.02, seed=1)
    return W.small_dambreak2d(l0=0.01, seed=2)


@pytest.mark.parametrize("dim", [3, 2])
def test_deck_loaders_match_reference(dim, tmp_path):
    mine, ref = _libs(dim)
    wl = _case(dim)
    cal = wl.write(str(tmp_path / "deck"))
    # comments, blank lines and an unknown key, which both loaders skip
    with open(os.path.join(tmp_path, "deck", "params.txt"), "a") as fh:
        fh.write("\n# a comment line\nnot_a_key 12\nrelaxation_coeff 0.25\n")
    SC = T.sim_config_type(dim)
    out = []
    for lib in (mine, ref):
        cfg = SC()
        lib.config_set_defaults(C.byref(cfg))
        assert lib.config_load_cal(cal.encode(), C.byref(cfg)) == 0
        assert lib.config_load_params(cfg.param_file, C.byref(cfg)) == 0
        out.append(bytes(cfg))
    out.append(bytes(CF.load_deck(cal, dim)))
    assert out[0] == out[1]
    assert out[2] == out[1]
    cfg = SC.from_buffer_copy(out[0])
    assert cfg.relaxation_coeff == 0.25 and cfg.particle_distance == wl.config().particle_distance


@pytest.mark.parametrize("dim", [3, 2])
def test_writers_match_reference(dim, tmp_path):
    mine, ref = _libs(dim)
    wl = _case(dim)
    hp = T.HostParticles(dim, wl.pos, wl.vel, wl.types)
    rng = np.random.default_rng(3)
    v = hp.view
    v["vel"] = rng.normal(0.0, 0.7, size=v["vel"].shape)
    v["pressure"] = rng.normal(0.0, 1500.0, size=hp.n)
    v["n"] = rng.uniform(10.0, 20.0, size=hp.n)
    v["type"][5] = 2      # a ghost: the writers skip it
    files = []
    for name, lib in (("mine", mine), ("ref", ref)):
        d = tmp_path / name
        d.mkdir()
        lib.output_csv(C.byref(hp.ps), 7, str(d).encode())
        lib.output_vtk(C.byref(hp.ps), 7, str(d).encode())
        files.append({f: (d / f).read_bytes() for f in sorted(os.listdir(d))})
    assert len(files[0]) == 2 and files[0].keys() == files[1].keys()
    for f in files[0]:
        assert files[0][f] == files[1][f], f
