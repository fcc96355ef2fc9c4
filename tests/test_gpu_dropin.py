"""The drop-in libraries (libmps3d.so / libmps2d.so): the reference's own
entry points, called exactly as the reference's main.c and simulation.c call
them, against the reference compiled from source (oracle/_ref).

Bit-exact: neighbour lists and cell chains, number density.  Tolerance
(stated per test): states after full steps, where the PPE solve's
floating-point noise enters."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import reference_lib
from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _dropin(dim):
    lib = C.CDLL(os.path.join(ROOT, "mps_b200", f"libmps{dim}d.so"))
    PS = C.POINTER(T.ParticleSystem)
    NL = C.POINTER(T.NeighborList)
    CL = C.POINTER(T.cell_list_type(dim))
    lib.cell_list_create.restype = CL
    lib.cell_list_create.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    lib.cell_list_free.argtypes = [CL]
    lib.neighbor_search_cell_linked_list.argtypes = [NL, PS, CL, C.c_double]
    lib.simulation_step.argtypes = [PS, NL, CL, C.c_int]
    lib.particle_system_calc_initial_params.argtypes = [PS]
    lib.calc_particle_number_density.argtypes = [PS, NL]
    lib.solve_pressure.argtypes = [PS, NL]
    lib.mps_dropin_release.argtypes = [PS]
    lib.mps_dropin_last_status.restype = C.c_int
    lib.mps_dropin_set_exit_on_error(0)
    return lib


def _cells(lib, n, re, cfg, dim):
    dmin = (C.c_double * dim)(*cfg.domain_min)
    dmax = (C.c_double * dim)(*cfg.domain_max)
    return lib.cell_list_create(n, re, C.cast(dmin, C.c_void_p), C.cast(dmax, C.c_void_p))


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("dim", [3, 2])
def test_dropin_steps_match_reference(dim):
    """simulation_run's call sequence through both libraries: n0/lambda and
    every neighbour list bit-exact; after 5 steps pressure within 1e-7 and
    positions within 1e-12 relative L2."""
    _cuda()
    kind = "3d" if dim == 3 else "2d"
    ref = reference_lib(kind)
    mine = _dropin(dim)
    wl = W.small_dambreak3d(l0=0.02, seed=21) if dim == 3 else W.small_dambreak2d(l0=0.01, seed=21)
    cfg = wl.config()
    re = CF.neighbor_radius(cfg)
    C.c_void_p.in_dll(mine, "g_config").value = C.addressof(cfg)
    ref.set_config(cfg)
    hm = T.HostParticles(dim, wl.pos, wl.vel, wl.types)
    hr = hm.copy()
    mine.particle_system_calc_initial_params(C.byref(hm.ps))
    ref.lib.particle_system_calc_initial_params(C.byref(hr.ps))
    assert (hm.ps.n0, hm.ps.lambda_) == (hr.ps.n0, hr.ps.lambda_)
    m = cfg.max_neighbors
    nlm, nlr = T.HostNeighborList(hm.n, m), T.HostNeighborList(hr.n, m)
    clm, clr = _cells(mine, hm.n, re, cfg, dim), ref.cell_list(hr.n, re, cfg)
    mine.neighbor_search_cell_linked_list(C.byref(nlm.nl), C.byref(hm.ps), clm, re)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nlr.nl), C.byref(hr.ps), clr, re)
    for step in range(1, 6):
        assert np.array_equal(nlm.count, nlr.count)
        for i in range(hm.n):
            c = nlm.count[i]
            assert np.array_equal(nlm.neighbors[i * m: i * m + c], nlr.neighbors[i * m: i * m + c])
        mine.simulation_step(C.byref(hm.ps), C.byref(nlm.nl), clm, step)
        ref.step(hr, nlr, clr, step)
        assert mine.mps_dropin_last_status() == 0
    hd = np.ctypeslib.as_array(clm.contents.head, shape=(clm.contents.total_cells,))
    hdr = np.ctypeslib.as_array(clr.contents.head, shape=(clr.contents.total_cells,))
    assert np.array_equal(hd, hdr)
    a, b = hm.view, hr.view
    assert np.array_equal(a["type"], b["type"])
    assert _rel(a["pressure"], b["pressure"]) < 1e-7
    assert _rel(a["pos"], b["pos"]) < 1e-12
    mine.mps_dropin_release(C.byref(hm.ps))
    mine.cell_list_free(clm)
    ref.lib.cell_list_free(clr)


def test_dropin_fine_grained_bitexact():
    """calc_particle_number_density and solve_pressure called one by one."""
    _cuda()
    ref = reference_lib("3d")
    mine = _dropin(3)
    wl = W.small_dambreak3d(l0=0.02, seed=22)
    cfg = wl.config()
    re = CF.neighbor_radius(cfg)
    C.c_void_p.in_dll(mine, "g_config").value = C.addressof(cfg)
    ref.set_config(cfg)
    hr = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    ref.lib.particle_system_calc_initial_params(C.byref(hr.ps))
    m = cfg.max_neighbors
    nl = T.HostNeighborList(hr.n, m)
    clr = ref.cell_list(hr.n, re, cfg)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nl.nl), C.byref(hr.ps), clr, re)
    for s in range(1, 3):
        ref.step(hr, nl, clr, s)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nl.nl), C.byref(hr.ps), clr, re)
    hm = hr.copy()
    ref.lib.calc_particle_number_density(C.byref(hr.ps), C.byref(nl.nl))
    mine.calc_particle_number_density(C.byref(hm.ps), C.byref(nl.nl))
    assert np.array_equal(hm.view["n"], hr.view["n"])
    ref.lib.solve_pressure(C.byref(hr.ps), C.byref(nl.nl))
    mine.solve_pressure(C.byref(hm.ps), C.byref(nl.nl))
    assert mine.mps_dropin_last_status() == 0
    assert _rel(hm.view["pressure"], hr.view["pressure"]) < 1e-8
    mine.mps_dropin_release(C.byref(hm.ps))
    ref.lib.cell_list_free(clr)


def test_cli_runs_deck_and_writes_reference_formats(tmp_path):
    """mps_sim3d <cal.txt>: the reference's CLI contract and output files."""
    _cuda()
    wl = W.small_dambreak3d(l0=0.025, seed=23, steps=6)
    wl.params["output_interval"] = "3"
    cal = wl.write(str(tmp_path / "deck"))
    exe = os.path.join(ROOT, "mps_b200", "mps_sim3d")
    r = subprocess.run([exe, cal], cwd=str(tmp_path / "deck"), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Simulation complete." in r.stdout
    out = tmp_path / "deck" / "output"
    for step in (0, 3, 6):
        csv = (out / f"output_{step:06d}.csv").read_text().splitlines()
        assert csv[0] == "x,y,z,vx,vy,vz,pressure,type"
        assert len(csv) - 1 == wl.n
        vtk = (out / f"output_{step:06d}.vtk").read_text().splitlines()
        assert vtk[:4] == ["# vtk DataFile Version 3.0", f"MPS 3D Simulation Step {step}", "ASCII",
                           "DATASET UNSTRUCTURED_GRID"]
    # step 0 equals the deck
    a = np.loadtxt(out / "output_000000.csv", delimiter=",", skiprows=1)
    assert np.allclose(a[:, :3], wl.pos, rtol=0, atol=1e-9)
