"""The reference's optional physics switches on the GPU, against the oracle.

The oracle's restatement of each switch is pinned bit for bit to the
reference build (tests/test_oracle_pin.py); here the CUDA path runs the
same step from the same state and list, through the C ABI:

  * ppe_type 1: the PPE diagonal scaled by c_ppe (pressure_solver.c:326-340,
    381-409);
  * cmps_gradient 1 and 2: the CMPS and Oochi pressure gradients
    (operators.c:158-168), the second without the P_min term;
  * surface_detection_method 1: the neighbour-count surface test
    (operators.c:226-267), with its N0 from the initial parameters;
  * hs_mode 1 with the negative-pressure clamp (pressure_solver.c:342-362,
    operators.c:188-199);
  * surface tension with wetting (operators.c:281-354, 2-D operators.c:
    231-309; coefficients of particle.c:185-211): the list radius grows to
    influence_radius_st, the explicit stage adds the potential forces.

Bit-exact: neighbour lists, number densities, neighbour counts, surface
flags, types, the PPE matrix and right-hand side; pressures within 1e-8
relative L2 (the solver's ordering), velocity 1e-10 and position 1e-14
after the step, as for the default switches (tests/test_gpu_parity.py).
The gradient stage alone, on identical pressures, is bit-exact too.
"""
import ctypes as C

import numpy as np
import pytest

from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W

pytestmark = pytest.mark.gpu

P_TOL, V_TOL, X_TOL = 1e-8, 1e-10, 1e-14

SWITCHES = {
    "ppe_type1": dict(ppe_type=1, c_ppe=1.01),
    "cmps1": dict(cmps_gradient=1),
    "cmps2_countsurf": dict(cmps_gradient=2, surface_detection_method=1),
    "hs1_clamp": dict(hs_mode=1, clamp_negative_pressure=1),
    "surface_tension": dict(surface_tension_enabled=1, wetting_angle_SL=60.0),
}


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _workload(dim, sw):
    if dim == 3:
        return W.small_dambreak3d(l0=0.02, seed=21, **sw)
    return W.small_dambreak2d(l0=0.01, seed=22, **sw)


def _moved(wl, orc, steps=2):
    """Initial parameters, the first list, and `steps` oracle steps, so the
    flow has started (non-zero gradients, some surface changes)."""
    cfg = wl.config()
    hp = T.HostParticles(wl.dim, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hp.n, cfg.max_neighbors)
    cl = orc.cell_list(hp.n, re, cfg)
    assert orc.search(nl, hp, cl, re) == 0
    for _ in range(steps):
        assert orc.step(hp, nl, cl, cfg) == 0
    return cfg, hp, nl, cl


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("name", sorted(SWITCHES))
def test_switch_step_matches_oracle(name, dim):
    _cuda()
    from mps_b200.session import Session
    from oracle.pyoracle import Oracle
    orc = Oracle(dim)
    wl = _workload(dim, SWITCHES[name])
    cfg, hp, nl, cl = _moved(wl, orc)
    m = cfg.max_neighbors
    hg = hp.copy()
    nb_prev, cnt_prev = nl.neighbors[: hp.n * m].copy(), nl.count[: hp.n].copy()
    assert orc.step(hp, nl, cl, cfg) == 0
    with Session(cfg, dim, hg.n) as s:
        s.upload(hg)
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.step_with_list(nb_prev, cnt_prev, m)
        g = s.download()
        nb, cnt = s.neighbor_list(m)
    o = hp.view
    assert np.array_equal(cnt, nl.count[: hp.n])
    for i in range(hp.n):
        assert np.array_equal(nb[i * m: i * m + cnt[i]], nl.neighbors[i * m: i * m + cnt[i]]), i
    for f in ("n", "on_surface", "type", "neighbor_count"):
        assert np.array_equal(g[f], o[f]), f
    assert _rel(g["pressure"], o["pressure"]) < P_TOL, _rel(g["pressure"], o["pressure"])
    assert _rel(g["vel"], o["vel"]) < V_TOL
    assert _rel(g["pos"], o["pos"]) < X_TOL
    if name == "hs1_clamp":
        # the clamp acts on fluid particles only (operators.c:188-199)
        assert np.all(g["pressure"][g["type"] == 0] >= 0.0)


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("name", sorted(SWITCHES))
def test_switch_ppe_bitexact(name, dim):
    """The PPE matrix and right-hand side of the switch, in the reference's
    numbering, bit for bit."""
    _cuda()
    from mps_b200.session import Session
    from oracle.pyoracle import Oracle
    orc = Oracle(dim)
    wl = _workload(dim, SWITCHES[name])
    cfg, hp, nl, cl = _moved(wl, orc)
    m = cfg.max_neighbors
    # the stage inputs the solve sees: a list of the current positions,
    # densities and flags
    assert orc.search(nl, hp, cl, CF.neighbor_radius(cfg)) == 0
    L = orc.lib
    L.oracle_number_density(C.byref(hp.ps), C.byref(nl.nl), C.byref(cfg))
    if cfg.surface_detection_method == 1:
        L.oracle_neighbor_count(C.byref(hp.ps), C.byref(nl.nl), C.byref(cfg))
        L.oracle_judge_free_surface_by_count(C.byref(hp.ps), cfg.surface_count_threshold)
    else:
        L.oracle_judge_free_surface(C.byref(hp.ps), cfg.surface_threshold)
    eq, rp, ci, va, b = orc.assemble(hp, nl, cfg)
    with Session(cfg, dim, hp.n) as s:
        s.upload(hp)
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.run_stage("solve_pressure", nl.neighbors[: hp.n * m], nl.count[: hp.n], m)
        geq, grp, gci, gva, gb = s.ppe()
    assert np.array_equal(geq, eq)
    assert np.array_equal(grp, rp)
    assert np.array_equal(gci, ci)
    assert np.array_equal(gva, va)
    assert np.array_equal(gb, b)


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("cmps", [1, 2])
def test_cmps_gradient_stage_bitexact(cmps, dim):
    """The gradient stage alone on identical pressures: CMPS (1) and Oochi
    (2) gradients give the oracle's accelerations, velocities and positions
    bit for bit."""
    _cuda()
    from mps_b200.session import Session
    from oracle.pyoracle import Oracle
    orc = Oracle(dim)
    wl = _workload(dim, {"cmps_gradient": cmps})
    cfg, hp, nl, cl = _moved(wl, orc)
    m = cfg.max_neighbors
    hg = hp.copy()
    orc.lib.oracle_pressure_gradient(C.byref(hp.ps), C.byref(nl.nl), C.byref(cfg))
    with Session(cfg, dim, hg.n) as s:
        s.upload(hg)
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.run_stage("gradient", nl.neighbors[: hp.n * m], nl.count[: hp.n], m)
        g = s.download()
    o = hp.view
    assert np.any(o["acc"] != hg.view["acc"])
    for f in ("acc", "vel", "pos", "pressure"):
        assert np.array_equal(g[f], o[f]), f


@pytest.mark.parametrize("dim", [3, 2])
def test_surface_tension_stages_bitexact(dim):
    """calc_surface_tension and calc_surface_tension_SL alone, on the same
    state and list, with the coefficients of the caller's particle system:
    accelerations bit for bit."""
    _cuda()
    from mps_b200.session import Session
    from oracle.pyoracle import Oracle
    orc = Oracle(dim)
    wl = _workload(dim, SWITCHES["surface_tension"])
    cfg, hp, nl, cl = _moved(wl, orc)
    assert hp.ps.C_LL > 0.0 and hp.ps.C_SL > 0.0
    m = cfg.max_neighbors
    L = orc.lib
    for stage, fn, coeff in (("surface_tension", L.oracle_surface_tension, hp.ps.C_LL),
                             ("surface_tension_sl", L.oracle_surface_tension_SL, hp.ps.C_SL)):
        ho = hp.copy()
        ho.view["acc"][:] = 0.0
        hg = ho.copy()
        fn(C.byref(ho.ps), C.byref(nl.nl), C.byref(cfg))
        with Session(cfg, dim, hg.n) as s:
            s.upload(hg)
            s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
            s.run_stage(stage, nl.neighbors[: hp.n * m], nl.count[: hp.n], m, arg=coeff)
            g = s.download()
        assert np.any(ho.view["acc"] != 0.0), stage
        assert np.array_equal(g["acc"], ho.view["acc"]), stage


@pytest.mark.parametrize("theta", [90.0, 60.0])
def test_friction_step_matches_oracle(theta):
    """The contact-line friction of the 3-D serial variant (mps_fluid3D
    operators.c:337-492; the oracle's restatement is pinned to that build by
    tests/test_oracle_pin.py): a full step from the same state and list,
    lists, densities, flags and types bit for bit, pressure within 1e-8,
    velocity 1e-10, position 1e-14."""
    _cuda()
    from mps_b200.session import Session
    from oracle.pyoracle import Oracle
    orc = Oracle(3)
    wl = W.small_dambreak3d(l0=0.02, seed=23, friction_enabled=1, wetting_angle_SL=theta)
    orc.set_friction(wl.config())
    try:
        cfg, hp, nl, cl = _moved(wl, orc)
        m = cfg.max_neighbors
        hg = hp.copy()
        nb_prev, cnt_prev = nl.neighbors[: hp.n * m].copy(), nl.count[: hp.n].copy()
        assert orc.step(hp, nl, cl, cfg) == 0
    finally:
        orc.set_friction(W.small_dambreak3d(l0=0.02, seed=23).config())
    with Session(cfg, 3, hg.n) as s:
        s.upload(hg)
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.step_with_list(nb_prev, cnt_prev, m)
        g = s.download()
    o = hp.view
    for f in ("n", "on_surface", "type"):
        assert np.array_equal(g[f], o[f]), f
    assert _rel(g["pressure"], o["pressure"]) < P_TOL, _rel(g["pressure"], o["pressure"])
    assert _rel(g["vel"], o["vel"]) < V_TOL
    assert _rel(g["pos"], o["pos"]) < X_TOL
