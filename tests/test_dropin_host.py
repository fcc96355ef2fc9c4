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


@pytest.mark.parametrize("dim", [3, 2])
def test_host_helpers_match_reference(dim, capfd):
    """kernel_weight(_derivative) over r from 0 (below the 0.01 l0 floor)
    past re, particle_system_create/add (including adds past the capacity),
    neighbor_list_create / neighbor_get, cell_list_create's grid and
    config_print's text: the same values and bytes as the reference's."""
    mine, ref = _libs(dim)
    SC = T.sim_config_type(dim)
    CL = T.cell_list_type(dim)
    PS, NL = C.POINTER(T.ParticleSystem), C.POINTER(T.NeighborList)
    keep = []
    for lib in (mine, ref):
        cfg = SC()
        lib.config_set_defaults(C.byref(cfg))
        cfg.particle_distance = 0.01
        keep.append(cfg)
        C.c_void_p.in_dll(lib, "g_config").value = C.addressof(cfg)
        for fn in ("kernel_weight", "kernel_weight_derivative"):
            getattr(lib, fn).restype = C.c_double
            getattr(lib, fn).argtypes = [C.c_double, C.c_double]
        lib.particle_system_create.restype = PS
        lib.particle_system_create.argtypes = [C.c_int]
        lib.particle_system_add.argtypes = [PS, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
        lib.particle_system_free.argtypes = [PS]
        lib.neighbor_list_create.restype = NL
        lib.neighbor_list_create.argtypes = [C.c_int, C.c_int]
        lib.neighbor_list_free.argtypes = [NL]
        lib.neighbor_get.argtypes = [NL, C.c_int, C.c_int]
        lib.cell_list_create.restype = C.POINTER(CL)
        lib.cell_list_create.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        lib.cell_list_free.argtypes = [C.POINTER(CL)]
        lib.config_print.argtypes = [C.POINTER(SC)]

    rs = np.concatenate([[0.0, 1e-6, 1e-4, 0.021, np.nextafter(0.021, 1.0), np.nextafter(0.021, 0.0)],
                         np.linspace(0.0, 0.04, 401)])
    for re in (0.021, 0.031):
        for fn in ("kernel_weight", "kernel_weight_derivative"):
            a = np.array([getattr(mine, fn)(float(r), re) for r in rs])
            b = np.array([getattr(ref, fn)(float(r), re) for r in rs])
            assert np.array_equal(a, b), (fn, re)

    rng = np.random.default_rng(4)
    pos = rng.normal(size=(8, dim))
    vel = rng.normal(size=(8, dim))
    item = T.particle_dtype(dim).itemsize
    seen = []
    for lib in (mine, ref):
        ps = lib.particle_system_create(6)
        rc = [lib.particle_system_add(ps, (C.c_double * dim)(*pos[k]), (C.c_double * dim)(*vel[k]), k % 4)
              for k in range(8)]
        s = ps.contents
        seen.append((rc, s.num, s.capacity, C.string_at(s.particles, s.num * item)))
        lib.particle_system_free(ps)
    assert seen[0] == seen[1]
    assert seen[0][0] == [0, 1, 2, 3, 4, 5, -1, -1]

    got = []
    for lib in (mine, ref):
        nl = lib.neighbor_list_create(5, 8)
        cnt = [nl.contents.count[i] for i in range(5)]
        for i in range(5):
            nl.contents.count[i] = i + 1
            for j in range(i + 1):
                nl.contents.neighbors[i * 8 + j] = 100 * i + j
        got.append((nl.contents.max_neighbors, cnt,
                    [lib.neighbor_get(nl, i, j) for i in range(5) for j in range(i + 1)]))
        lib.neighbor_list_free(nl)
    assert got[0] == got[1] and got[0][1] == [0] * 5

    lo = (C.c_double * dim)(*([-0.013] * dim))
    hi = (C.c_double * dim)(*[1.6, 0.6, 0.6][:dim])
    grids = []
    for lib in (mine, ref):
        cl = lib.cell_list_create(1000, 0.031, C.cast(lo, C.c_void_p), C.cast(hi, C.c_void_p))
        c = cl.contents
        grids.append(tuple(getattr(c, f) for f, _ in CL._fields_ if f not in ("head", "next", "origin"))
                     + tuple(c.origin))
        lib.cell_list_free(cl)
    assert grids[0] == grids[1]

    # the configuration report: defaults, then every optional line switched on
    libc = C.CDLL(None)
    for switches in ({}, dict(ppe_type=1, surface_detection_method=1, surface_tension_enabled=1, cmps_gradient=1,
                              clamp_negative_pressure=1, use_analytical_lambda=1, hs_mode=1,
                              surface_tension_coeff=0.0728, influence_radius_st=0.031)):
        texts = []
        for lib, cfg in zip((mine, ref), keep):
            for k, v in switches.items():
                setattr(cfg, k, v)
            capfd.readouterr()
            lib.config_print(C.byref(cfg))
            libc.fflush(None)
            texts.append(capfd.readouterr().out)
        assert texts[0] == texts[1] and len(texts[0]) > 200, switches
