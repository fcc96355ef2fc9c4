"""Parity at the benchmarked sizes (slow: a few minutes, most of it the
reference's own CPU step).

c1 single step, 3-D dam break at l0 = 0.005 m (1,170,276 particles), the
GPU step through the C ABI (mps_step_with_list: the reference's previous
list drives the explicit stage) against the reference compiled from its
own sources (oracle/_ref) on the same initial state:

  * the new neighbour list: every particle's count, and the members and
    order of 50,000 sampled rows, bit for bit; the cell chains (head/next)
    bit for bit;
  * number densities, surface flags and types bit for bit;
  * pressure within 1e-8 relative L2, velocity 1e-10, position 1e-14 (the
    PPE solve's ordering, as at small sizes);
  * the PPE matrix and right-hand side of the step's state, in the
    reference's numbering, bit for bit against the oracle's assembly (the
    reference does not expose its matrix; the oracle's is pinned to it at
    small sizes by the pressures it produces).

c2 mixed form over 20 steps, 3-D dam break at l0 = 0.0035 m (2,854,670
particles): the mixed-precision form against the FP64 form from one
initial state; the stated tolerance is the pressure criterion of the mixed
form, relative L2 <= 1e-4, with velocity <= 1e-5 and position <= 1e-8 over
the fluid, and no type differs.
"""
import ctypes as C

import numpy as np
import pytest

from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def test_c1_step_against_reference_build():
    _cuda()
    from conftest import reference_lib
    from mps_b200.session import Session
    from oracle.pyoracle import Oracle
    ref = reference_lib("3d")
    orc = Oracle(3)
    wl = W.dambreak("c1", seed=1000)
    cfg = wl.config()
    m = cfg.max_neighbors
    re = CF.neighbor_radius(cfg)
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)       # bit-identical to the reference's O(N^2) loop
    ref.set_config(cfg)
    nl = T.HostNeighborList(hp.n, m)
    cl = ref.cell_list(hp.n, re, cfg)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nl.nl), C.byref(hp.ps), cl, re)
    nb_prev, cnt_prev = nl.neighbors[: hp.n * m].copy(), nl.count[: hp.n].copy()
    hg = hp.copy()
    # the step's PPE inputs, from the oracle's stages on a copy
    ho = hp.copy()
    L = orc.lib
    ho_nl = T.HostNeighborList(hp.n, m)
    ho_nl.neighbors[:] = nl.neighbors
    ho_nl.count[:] = nl.count
    ocl = orc.cell_list(hp.n, re, cfg)
    fl = ho.view["type"] == 0
    ho.view["acc"][:] = 0.0
    ho.view["acc"][fl] = np.array(cfg.gravity[:3])
    L.oracle_viscosity(C.byref(ho.ps), C.byref(ho_nl.nl), C.byref(cfg))
    f = ho.view["type"] == 0
    ho.view["vel"][f] += cfg.dt * ho.view["acc"][f]
    ho.view["pos"][f] += cfg.dt * ho.view["vel"][f]
    assert L.oracle_collision(C.byref(ho.ps), C.byref(ho_nl.nl), C.byref(cfg)) == 0
    assert orc.search(ho_nl, ho, ocl, re) == 0
    L.oracle_number_density(C.byref(ho.ps), C.byref(ho_nl.nl), C.byref(cfg))
    L.oracle_judge_free_surface(C.byref(ho.ps), cfg.surface_threshold)
    eq, rp, ci, va, b = orc.assemble(ho, ho_nl, cfg)
    # the reference's step
    ref.step(hp, nl, cl, 1)
    o = hp.view
    with Session(cfg, 3, hg.n) as s:
        s.upload(hg)
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.step_with_list(nb_prev, cnt_prev, m)
        g = s.download()
        gcnt = s.neighbor_counts(m)
        gnb, gcnt2 = s.neighbor_list(m)
        head, nxt = s.cell_links(cl.contents.total_cells)
        # the PPE of the step's state: the stage on the oracle's mid-step state
        s.upload(ho)
        s.run_stage("solve_pressure", ho_nl.neighbors[: hp.n * m], ho_nl.count[: hp.n], m)
        geq, grp, gci, gva, gb = s.ppe()
    assert np.array_equal(gcnt, nl.count[: hp.n]) and np.array_equal(gcnt2, gcnt)
    rows = np.random.default_rng(3).choice(hp.n, size=50_000, replace=False)
    for i in rows:
        assert np.array_equal(gnb[i * m: i * m + gcnt[i]], nl.neighbors[i * m: i * m + gcnt[i]]), i
    tc = cl.contents.total_cells
    assert np.array_equal(head, np.ctypeslib.as_array(cl.contents.head, shape=(tc,)))
    assert np.array_equal(nxt, np.ctypeslib.as_array(cl.contents.next, shape=(hp.n,)))
    for fld in ("n", "on_surface", "type"):
        assert np.array_equal(g[fld], o[fld]), fld
    assert _rel(g["pressure"], o["pressure"]) < 1e-8, _rel(g["pressure"], o["pressure"])
    assert _rel(g["vel"], o["vel"]) < 1e-10
    assert _rel(g["pos"], o["pos"]) < 1e-14
    assert np.array_equal(geq, eq)
    assert np.array_equal(grp, rp)
    assert np.array_equal(gci, ci)
    assert np.array_equal(gva, va)
    assert np.array_equal(gb, b)
    ref.lib.cell_list_free(cl)


def test_c2_mixed_form_against_fp64_20_steps():
    _cuda()
    from mps_b200 import _lib
    from mps_b200.session import start
    wl = W.dambreak("c2", seed=1001)
    cfg = wl.config()
    h64 = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    a = start(cfg, 3, h64)
    ga = None
    try:
        a.step(20)
        ga = a.download()
    finally:
        a.close()
    h32 = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    b = start(cfg, 3, h32, precision=_lib.PREC_MIXED)
    try:
        b.step(20)
        gb = b.download()
        mb = b.metrics()
    finally:
        b.close()
    assert mb["converged"] == 1
    assert np.array_equal(ga["type"], gb["type"])
    fl = ga["type"] == 0
    ep = _rel(gb["pressure"], ga["pressure"])
    ev = _rel(gb["vel"][fl], ga["vel"][fl])
    ex = _rel(gb["pos"][fl], ga["pos"][fl])
    print(f"c2, 20 steps, mixed vs FP64: pressure {ep:.3e}, velocity {ev:.3e}, position {ex:.3e}")
    assert ep <= 1e-4, ep
    assert ev <= 1e-5, ev
    assert ex <= 1e-8, ex
