"""Pins the CPU oracle (oracle/mps_oracle.c) before anything is checked against it.

1. Against the reference compiled from its own sources (oracle/_ref): every
   field of every particle is bit-identical after each of several full steps,
   in 3-D and 2-D, and the initial n0/lambda agree.
2. Against the reference's shipped 3-D dam-break trajectory
   (tests/golden/dambreak3d_golden.npz, made by tests/golden/make_golden.py):
   100 steps of the example deck reproduce every fluid row of
   output_000100.csv at the file's %.8e precision.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import REF_DIR, reference_lib
from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W

FIELDS = ["pos", "vel", "acc", "pressure", "n", "type", "on_surface"]
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "dambreak3d_golden.npz")


def _setup(orc, wl, cfg):
    hp = T.HostParticles(wl.dim, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hp.n, cfg.max_neighbors)
    cl = orc.cell_list(hp.n, re, cfg)
    assert orc.search(nl, hp, cl, re) == 0
    return hp, nl, cl


@pytest.mark.parametrize("dim,kind", [(3, "3d"), (2, "2d")])
def test_oracle_bitexact_vs_reference_steps(dim, kind, oracle3, oracle2):
    orc = oracle3 if dim == 3 else oracle2
    ref = reference_lib(kind)
    wl = W.small_dambreak3d(l0=0.02, seed=3) if dim == 3 else W.small_dambreak2d(l0=0.02, seed=3)
    cfg = wl.config()
    hp_o, nl_o, cl_o = _setup(orc, wl, cfg)
    hp_r = T.HostParticles(dim, wl.pos, wl.vel, wl.types)
    ref.set_config(cfg)
    ref.lib.particle_system_calc_initial_params(C.byref(hp_r.ps))
    assert hp_o.ps.n0 == hp_r.ps.n0 and hp_o.ps.lambda_ == hp_r.ps.lambda_
    re = CF.neighbor_radius(cfg)
    nl_r = T.HostNeighborList(hp_r.n, cfg.max_neighbors)
    cl_r = ref.cell_list(hp_r.n, re, cfg)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nl_r.nl), C.byref(hp_r.ps), cl_r, re)
    assert np.array_equal(nl_o.count, nl_r.count)
    for s in range(1, 5):
        assert orc.step(hp_o, nl_o, cl_o, cfg) == 0
        ref.step(hp_r, nl_r, cl_r, s)
        for f in FIELDS:
            assert np.array_equal(hp_o.view[f], hp_r.view[f]), (s, f)
        assert np.array_equal(nl_o.count, nl_r.count)
    ref.lib.cell_list_free(cl_r)


@pytest.mark.parametrize("hs,clamp,cmps,surf", [(1, 1, 0, 0), (0, 0, 1, 0), (0, 0, 2, 1)])
def test_oracle_bitexact_switches(hs, clamp, cmps, surf, oracle3):
    """The optional physics switches restated in the oracle also match."""
    ref = reference_lib("3d")
    wl = W.small_dambreak3d(l0=0.025, seed=5, hs_mode=hs, clamp_negative_pressure=clamp,
                            cmps_gradient=cmps, surface_detection_method=surf)
    cfg = wl.config()
    hp_o, nl_o, cl_o = _setup(oracle3, wl, cfg)
    hp_r = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    ref.set_config(cfg)
    ref.lib.particle_system_calc_initial_params(C.byref(hp_r.ps))
    assert hp_o.ps.n0_count == hp_r.ps.n0_count
    re = CF.neighbor_radius(cfg)
    nl_r = T.HostNeighborList(hp_r.n, cfg.max_neighbors)
    cl_r = ref.cell_list(hp_r.n, re, cfg)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nl_r.nl), C.byref(hp_r.ps), cl_r, re)
    for s in range(1, 4):
        oracle3.step(hp_o, nl_o, cl_o, cfg)
        ref.step(hp_r, nl_r, cl_r, s)
        for f in FIELDS + ["neighbor_count"]:
            assert np.array_equal(hp_o.view[f], hp_r.view[f]), (s, f)
    ref.lib.cell_list_free(cl_r)


def test_initial_params_cells_equal_all_pairs(oracle3, oracle2):
    for orc, wl in ((oracle3, W.small_dambreak3d(l0=0.02, seed=9, surface_detection_method=1)),
                    (oracle2, W.small_dambreak2d(l0=0.02, seed=9, surface_detection_method=1))):
        cfg = wl.config()
        a = T.HostParticles(wl.dim, wl.pos, wl.vel, wl.types)
        b = a.copy()
        orc.initial_params(a, cfg, cells=True)
        orc.initial_params(b, cfg, cells=False)
        assert (a.ps.n0, a.ps.lambda_, a.ps.n0_count) == (b.ps.n0, b.ps.lambda_, b.ps.n0_count)


def test_analytic_lambda(oracle3):
    wl = W.small_dambreak3d(l0=0.02, use_analytical_lambda=1)
    cfg = wl.config()
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    oracle3.initial_params(hp, cfg)
    re = cfg.influence_radius_lap
    assert hp.ps.lambda_ == re * re * 3.0 * 2.0 / (4.0 * 5.0)


def test_ppe_matrix_known_answers(oracle3):
    """Symmetric, positive diagonal, unknowns = interior fluid + wall."""
    wl = W.small_dambreak3d(l0=0.02, seed=1)
    cfg = wl.config()
    hp, nl, cl = _setup(oracle3, wl, cfg)
    oracle3.step(hp, nl, cl, cfg)
    eq, rp, ci, va, b = oracle3.assemble(hp, nl, cfg)
    v = hp.view
    expect = int(((v["type"] == 0) & (v["on_surface"] == 0)).sum() + (v["type"] == 1).sum())
    assert rp.shape[0] - 1 == expect
    n_eq = expect
    rows = np.repeat(np.arange(n_eq), np.diff(rp))
    assert np.all(np.diff(ci)[np.diff(rows) == 0] > 0)      # sorted, unique columns
    import scipy.sparse as sp
    A = sp.csr_matrix((va, ci, rp), shape=(n_eq, n_eq))
    assert abs(A - A.T).max() == 0.0
    assert np.all(A.diagonal() > 0)


def test_generator_matches_reference_example_deck():
    path = os.path.join(REF_DIR or "", "mps_fluid3D_parallel", "examples", "dambreak", "particles.txt")
    if not REF_DIR or not os.path.exists(path):
        pytest.skip("reference example deck not mounted")
    wl = W.example_dambreak3d()
    lines = [l for l in open(path).read().splitlines() if l and not l.startswith("#")][1:]
    mine = ["%.8e %.8e %.8e %.8e %.8e %.8e %d" % (*wl.pos[i], *wl.vel[i], wl.types[i]) for i in range(wl.n)]
    assert lines == mine


def test_oracle_reproduces_shipped_trajectory(oracle3):
    gold = np.load(GOLDEN)
    wl = W.example_dambreak3d()
    cfg = wl.config()
    step0 = gold["step0"]
    assert np.array_equal(step0[:, :3], wl.pos) and np.array_equal(step0[:, 7], wl.types)
    hp, nl, cl = _setup(oracle3, wl, cfg)
    for _ in range(100):
        assert oracle3.step(hp, nl, cl, cfg) == 0
    v = hp.view
    keep = v["type"] != 2
    mine = np.column_stack([v["pos"], v["vel"], v["pressure"], v["type"]])[keep]
    g = gold["step100"]
    assert mine.shape == g.shape
    as_text = np.vectorize(lambda x: "%.8e" % x)
    fluid = g[:, 7] == 0
    assert np.array_equal(as_text(mine[fluid, :7]), as_text(g[fluid, :7]))
    # Wall pressures: the shipped file was written on another CPU (FMA
    # contraction); they agree to the 8th significant digit.
    rel = np.abs(mine[:, 6] - g[:, 6]) / np.maximum(np.abs(g[:, 6]), 1.0)
    assert rel.max() < 1e-7


@pytest.mark.parametrize("dim,kind,theta", [(3, "3d", 90.0), (3, "3d", 60.0), (2, "2d", 60.0)])
def test_oracle_bitexact_surface_tension(dim, kind, theta, oracle3, oracle2):
    """Surface tension (3P operators.c:281-354, 2D operators.c:231-309) with
    its calibrated coefficients (particle.c:185-211): C_LL and C_SL equal the
    reference's, and so does every field after several steps; the C ABI's
    mps_surface_tension_coeffs gives the same coefficients."""
    from mps_b200 import _lib
    ref = reference_lib(kind)
    orc = oracle3 if dim == 3 else oracle2
    sw = dict(surface_tension_enabled=1, surface_tension_coeff=0.0728, surface_tension_re_ratio=3.2,
              wetting_angle_SL=theta)
    wl = (W.small_dambreak3d(l0=0.025, seed=7, **sw) if dim == 3 else W.small_dambreak2d(l0=0.02, seed=7, **sw))
    cfg = wl.config()
    assert cfg.surface_tension_enabled == 1 and cfg.influence_radius_st > cfg.influence_radius_lap
    hp_o, nl_o, cl_o = _setup(orc, wl, cfg)
    hp_r = T.HostParticles(dim, wl.pos, wl.vel, wl.types)
    ref.set_config(cfg)
    ref.lib.particle_system_calc_initial_params(C.byref(hp_r.ps))
    assert hp_o.ps.C_LL == hp_r.ps.C_LL and hp_o.ps.C_LL > 0.0
    assert hp_o.ps.C_SL == hp_r.ps.C_SL
    lib = _lib.load()
    cll, csl = C.c_double(), C.c_double()
    p = _lib.params_from_config(cfg, dim)
    assert lib.mps_surface_tension_coeffs(C.byref(p), C.byref(cll), C.byref(csl)) == 0
    assert (cll.value, csl.value) == (hp_r.ps.C_LL, hp_r.ps.C_SL)
    re = CF.neighbor_radius(cfg)
    nl_r = T.HostNeighborList(hp_r.n, cfg.max_neighbors)
    cl_r = ref.cell_list(hp_r.n, re, cfg)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nl_r.nl), C.byref(hp_r.ps), cl_r, re)
    for s in range(1, 4):
        assert orc.step(hp_o, nl_o, cl_o, cfg) == 0
        ref.step(hp_r, nl_r, cl_r, s)
        for f in FIELDS:
            assert np.array_equal(hp_o.view[f], hp_r.view[f]), (s, f)
        assert np.array_equal(nl_o.count, nl_r.count)
    ref.lib.cell_list_free(cl_r)


@pytest.mark.parametrize("theta", [90.0, 60.0])
def test_oracle_bitexact_friction(theta, oracle3):
    """The hybrid friction of the 3-D serial variant (mps_fluid3D
    operators.c:337-492, applied between the velocity and position updates,
    simulation.c:52-53): the oracle with its friction parameters set equals
    the serial reference build (oracle/_ref/libref3s.so, its own SimConfig
    layout) field for field over several steps, and friction changes the
    velocities against a run without it."""
    ref = reference_lib("3s")
    sw = dict(friction_enabled=1, wetting_angle_SL=theta, friction_velocity_threshold=0.01)
    wl = W.small_dambreak3d(l0=0.025, seed=8, **sw)
    cfg = wl.config()
    assert cfg.friction_enabled == 1
    oracle3.set_friction(cfg)
    try:
        hp_o, nl_o, cl_o = _setup(oracle3, wl, cfg)
        hp_r = T.HostParticles(3, wl.pos, wl.vel, wl.types)
        ref.set_config(cfg)
        ref.lib.particle_system_calc_initial_params(C.byref(hp_r.ps))
        re = CF.neighbor_radius(cfg)
        nl_r = T.HostNeighborList(hp_r.n, cfg.max_neighbors)
        cl_r = ref.cell_list(hp_r.n, re, cfg)
        ref.lib.neighbor_search_cell_linked_list(C.byref(nl_r.nl), C.byref(hp_r.ps), cl_r, re)
        for s in range(1, 4):
            assert oracle3.step(hp_o, nl_o, cl_o, cfg) == 0
            ref.step(hp_r, nl_r, cl_r, s)
            for f in FIELDS:
                assert np.array_equal(hp_o.view[f], hp_r.view[f]), (s, f)
        ref.lib.cell_list_free(cl_r)
        oracle3.set_friction(W.small_dambreak3d(l0=0.025, seed=8).config())
        hp_n, nl_n, cl_n = _setup(oracle3, wl, cfg)
        for s in range(1, 4):
            assert oracle3.step(hp_n, nl_n, cl_n, cfg) == 0
        assert not np.array_equal(hp_n.view["vel"], hp_o.view["vel"])
    finally:
        oracle3.set_friction(W.small_dambreak3d(l0=0.025, seed=8).config())
