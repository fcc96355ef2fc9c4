"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

Bit-exact for identical input states: neighbour sets (members and list
order), cell indices, cell chains, n0/lambda/N0, number densities, surface
flags, every operator output (viscosity, collision, gradient, neighbour
count), the PPE matrix and right-hand side in the reference's numbering.

Within tolerance: pressures after the PPE solve (relative L2 <= 1e-8; the
GPU uses a block-colour IC(0) and parallel reductions, so the converged
solution differs from the reference's only at the solver's floating-point
noise), and whole-step states (same bound on pressure, 1e-10 on velocity
and 1e-14 on position).
"""
import numpy as np
import pytest

from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W

pytestmark = pytest.mark.gpu

P_TOL = 1e-8     # pressure relative L2 after one solve / one step
V_TOL = 1e-10    # velocity relative L2 after one step
X_TOL = 1e-14    # position relative L2 after one step


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _oracle(dim):
    from oracle.pyoracle import Oracle
    return Oracle(dim)


def _prepare(wl, orc):
    cfg = wl.config()
    hp = T.HostParticles(wl.dim, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hp.n, cfg.max_neighbors)
    cl = orc.cell_list(hp.n, re, cfg)
    assert orc.search(nl, hp, cl, re) == 0
    return cfg, hp, nl, cl


def _session(cfg, dim, hp, **kw):
    from mps_b200.session import Session
    s = Session(cfg, dim, hp.n, **kw)
    s.upload(hp)
    return s


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _lists_equal(nb_a, cnt_a, nl_b, n, m):
    if not np.array_equal(cnt_a, nl_b.count[:n]):
        return False
    for i in range(n):
        if not np.array_equal(nb_a[i * m: i * m + cnt_a[i]], nl_b.neighbors[i * m: i * m + cnt_a[i]]):
            return False
    return True


CASES = [
    ("3d-small", lambda: W.small_dambreak3d(l0=0.02, seed=1)),
    ("2d-small", lambda: W.small_dambreak2d(l0=0.01, seed=2)),
    ("3d-c1geom-l0.02", lambda: W.dambreak("c1", l0=0.02, seed=3)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_neighbor_search_bitexact(name, make):
    _cuda()
    wl = make()
    orc = _oracle(wl.dim)
    cfg, hp, nl, cl = _prepare(wl, orc)
    with _session(cfg, wl.dim, hp) as s:
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.neighbor_search()
        nb, cnt = s.neighbor_list(cfg.max_neighbors)
        assert _lists_equal(nb, cnt, nl, hp.n, cfg.max_neighbors)
        # cell index as the reference computes it
        cell = s.cell_index()
        head, nxt = s.cell_links(cl.total_cells)
    ref_head = np.ctypeslib.as_array(cl.head, shape=(cl.total_cells,))
    ref_next = np.ctypeslib.as_array(cl.next, shape=(hp.n,))
    assert np.array_equal(head, ref_head)
    assert np.array_equal(nxt, ref_next)
    # cells from the chains
    ref_cell = np.full(hp.n, -1, dtype=np.int32)
    for c in np.nonzero(ref_head >= 0)[0]:
        j = ref_head[c]
        while j >= 0:
            ref_cell[j] = c
            j = ref_next[j]
    assert np.array_equal(cell, ref_cell)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_initial_params_bitexact(name, make):
    _cuda()
    wl = make()
    orc = _oracle(wl.dim)
    cfg = wl.config()
    cfg.surface_detection_method = 1
    hp = T.HostParticles(wl.dim, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)
    with _session(cfg, wl.dim, hp) as s:
        n0, lam, n0c = s.compute_initial_params()
    assert (n0, lam, n0c) == (hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)


def _moved_state(wl, orc, steps=2, research=False):
    """A state after a few oracle steps (non-trivial velocities, pressures).
    research: rebuild the list at the final positions (what solve_pressure sees)."""
    cfg, hp, nl, cl = _prepare(wl, orc)
    for _ in range(steps):
        assert orc.step(hp, nl, cl, cfg) == 0
    if research:
        assert orc.search(nl, hp, cl, CF.neighbor_radius(cfg)) == 0
    return cfg, hp, nl, cl


STAGE_CASES = [
    ("3d", lambda: W.small_dambreak3d(l0=0.02, seed=4)),
    ("2d", lambda: W.small_dambreak2d(l0=0.01, seed=5)),
]


@pytest.mark.parametrize("name,make", STAGE_CASES, ids=[c[0] for c in STAGE_CASES])
def test_operator_stages_bitexact(name, make):
    """Each operator on the same state and list gives the oracle's bits."""
    import ctypes as C
    _cuda()
    wl = make()
    orc = _oracle(wl.dim)
    cfg, hp, nl, cl = _moved_state(wl, orc)
    m = cfg.max_neighbors
    L = orc.lib
    for stage, run in [
        ("density", lambda h: L.oracle_number_density(C.byref(h.ps), C.byref(nl.nl), C.byref(cfg))),
        ("viscosity", lambda h: L.oracle_viscosity(C.byref(h.ps), C.byref(nl.nl), C.byref(cfg))),
        ("gradient", lambda h: L.oracle_pressure_gradient(C.byref(h.ps), C.byref(nl.nl), C.byref(cfg))),
        ("neighbor_count", lambda h: L.oracle_neighbor_count(C.byref(h.ps), C.byref(nl.nl), C.byref(cfg))),
        ("collision", lambda h: L.oracle_collision(C.byref(h.ps), C.byref(nl.nl), C.byref(cfg))),
    ]:
        ho = hp.copy()
        # make collisions happen: push a few fluid particles onto neighbours
        if stage == "collision":
            f = np.nonzero(ho.view["type"] == 0)[0][:50]
            ho.view["vel"][f] += 0.3
            ho.view["pos"][f] += 0.4 * cfg.particle_distance
        hg = ho.copy()
        run(ho)
        with _session(cfg, wl.dim, hg) as s:
            s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
            s.run_stage(stage, nl.neighbors[: hp.n * m], nl.count[: hp.n], m)
            g = s.download()
        o = ho.view
        for f in ("pos", "vel", "acc", "pressure", "n", "neighbor_count", "type", "on_surface"):
            assert np.array_equal(g[f], o[f]), (stage, f)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_ppe_matrix_bitexact_and_pressure(name, make):
    _cuda()
    wl = make()
    orc = _oracle(wl.dim)
    cfg, hp, nl, cl = _moved_state(wl, orc, steps=1, research=True)
    m = cfg.max_neighbors
    eq, rp, ci, va, b = orc.assemble(hp, nl, cfg)
    ho = hp.copy()
    import ctypes as C
    iters = orc.lib.oracle_solve_pressure(C.byref(ho.ps), C.byref(nl.nl), C.byref(cfg))
    with _session(cfg, wl.dim, hp) as s:
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.run_stage("solve_pressure", nl.neighbors[: hp.n * m], nl.count[: hp.n], m)
        geq, grp, gci, gva, gb = s.ppe()
        g = s.download()
        met = s.metrics()
    assert np.array_equal(geq, eq)
    assert np.array_equal(grp, rp)
    assert np.array_equal(gci, ci)
    assert np.array_equal(gva, va)
    assert np.array_equal(gb, b)
    assert _rel(g["pressure"], ho.view["pressure"]) < P_TOL
    assert met["converged"] == 1
    # iteration counts of the two orderings stay in the same range
    assert 0.5 * iters <= met["ppe_iterations"] <= 2.0 * iters + 5


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_full_step_with_reference_list(name, make):
    """simulation_step semantics: the previous step's list drives the explicit stage."""
    _cuda()
    wl = make()
    orc = _oracle(wl.dim)
    cfg, hp, nl, cl = _moved_state(wl, orc, steps=1)
    m = cfg.max_neighbors
    hg = hp.copy()
    nb_prev, cnt_prev = nl.neighbors[: hp.n * m].copy(), nl.count[: hp.n].copy()
    assert orc.step(hp, nl, cl, cfg) == 0
    with _session(cfg, wl.dim, hg) as s:
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.step_with_list(nb_prev, cnt_prev, m)
        g = s.download()
        nb, cnt = s.neighbor_list(m)
    o = hp.view
    assert _lists_equal(nb, cnt, nl, hp.n, m)
    for f in ("n", "on_surface", "type"):
        assert np.array_equal(g[f], o[f]), f
    assert _rel(g["pressure"], o["pressure"]) < P_TOL
    assert _rel(g["vel"], o["vel"]) < V_TOL
    assert _rel(g["pos"], o["pos"]) < X_TOL


@pytest.mark.parametrize("name,make", CASES[:2], ids=[c[0] for c in CASES[:2]])
def test_device_resident_steps_match_list_steps(name, make):
    """mps_step (cell structure kept on the device) equals step_with_list bit for bit."""
    _cuda()
    wl = make()
    orc = _oracle(wl.dim)
    cfg, hp, nl, cl = _prepare(wl, orc)
    m = cfg.max_neighbors
    with _session(cfg, wl.dim, hp) as a, _session(cfg, wl.dim, hp) as b:
        for s in (a, b):
            s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
            s.neighbor_search()
        for _ in range(3):
            a.step(1)
            nbp, cntp = b.neighbor_list(m)
            state = b.download()
            hb = T.HostParticles(wl.dim, state["pos"], state["vel"], state["type"])
            hb.arr[: hp.n] = state
            b.upload(hb)
            b.step_with_list(nbp, cntp, m)
        ga, gb = a.download(), b.download()
    for f in ("pos", "vel", "acc", "pressure", "n", "type", "on_surface"):
        assert np.array_equal(ga[f], gb[f]), f


def test_multistep_trajectory_3d():
    """20 device-resident steps against 20 oracle steps."""
    _cuda()
    wl = W.small_dambreak3d(l0=0.02, seed=6)
    orc = _oracle(3)
    cfg, hp, nl, cl = _prepare(wl, orc)
    hg = hp.copy()
    from mps_b200.session import start
    s = start(cfg, 3, hg)
    for _ in range(20):
        assert orc.step(hp, nl, cl, cfg) == 0
    s.step(20)
    g = s.download()
    s.close()
    o = hp.view
    assert np.array_equal(g["type"], o["type"])
    assert _rel(g["pressure"], o["pressure"]) < 1e-6
    assert _rel(g["pos"], o["pos"]) < 1e-12


def test_pinned_host_list_matches_pageable_list():
    """A neighbour list in page-locked host memory (read in place by the
    gather kernel) drives the same step as the same list in pageable memory
    (pitched copy), bit for bit; an out-of-range index in it is reported as
    an error, not followed."""
    _cuda()
    import torch
    from mps_b200 import _lib
    wl = W.small_dambreak3d(l0=0.02, seed=6)
    orc = _oracle(3)
    cfg, hp, nl, cl = _moved_state(wl, orc, steps=1)
    m = cfg.max_neighbors
    nb_prev, cnt_prev = nl.neighbors[: hp.n * m].copy(), nl.count[: hp.n].copy()
    nb_pin = torch.empty(hp.n * m, dtype=torch.int32, pin_memory=True).numpy()
    cnt_pin = torch.empty(hp.n, dtype=torch.int32, pin_memory=True).numpy()
    nb_pin[:] = nb_prev
    cnt_pin[:] = cnt_prev
    outs = []
    for nb, cnt in ((nb_prev, cnt_prev), (nb_pin, cnt_pin)):
        with _session(cfg, 3, hp.copy()) as s:
            s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
            s.step_with_list(nb, cnt, m)
            outs.append((s.download(), s.neighbor_list(m)))
    (ga, (nba, ca)), (gb, (nbb, cb)) = outs
    for f in ("pos", "vel", "acc", "pressure", "n", "type", "on_surface"):
        assert np.array_equal(ga[f], gb[f]), f
    assert np.array_equal(ca, cb)
    assert np.array_equal(nba, nbb)
    i = int(np.nonzero(cnt_pin > 0)[0][0])
    nb_pin[i * m] = hp.n + 5
    with _session(cfg, 3, hp.copy()) as s:
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        with pytest.raises(_lib.MpsError):
            s.step_with_list(nb_pin, cnt_pin, m)


def test_neighbor_overflow_reported():
    """max_neighbors too small: an error code, as the reference's exit(1)."""
    _cuda()
    from mps_b200 import _lib
    from mps_b200.session import Session
    wl = W.small_dambreak3d(l0=0.02, seed=7, max_neighbors=40)
    cfg = wl.config()
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    with Session(cfg, 3, hp.n) as s:
        s.upload(hp)
        s.compute_initial_params()
        with pytest.raises(_lib.MpsError) as e:
            s.neighbor_search()
        assert e.value.code == -4


def test_golden_trajectory_gpu():
    """The reference's example deck, 100 GPU steps vs its shipped output."""
    _cuda()
    import os
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "dambreak3d_golden.npz"))["step100"]
    wl = W.example_dambreak3d()
    cfg = wl.config()
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    from mps_b200.session import start
    s = start(cfg, 3, hp)
    s.step(100)
    g = s.download()
    s.close()
    keep = g["type"] != 2
    mine = np.column_stack([g["pos"], g["vel"], g["pressure"], g["type"]])[keep]
    assert mine.shape == gold.shape
    fluid = gold[:, 7] == 0
    # %.8e in the file: 5e-9 relative is its rounding
    assert _rel(mine[fluid, :3], gold[fluid, :3]) < 1e-8
    assert _rel(mine[fluid, 3:6], gold[fluid, 3:6]) < 1e-6
    assert _rel(mine[:, 6], gold[:, 6]) < 1e-6


@pytest.mark.parametrize("steps", [1, 20])
def test_mixed_precision_against_fp64(steps):
    """The mixed form (PPE matrix and IC(0) factor stored in FP32, FP64
    vectors, reliable updates against the FP64 matrix) stays within the
    1e-4 pressure relative-L2 target of the FP64 path, from the same state,
    and ends its solves at the residual level the FP64 path reaches: every
    step's true residual ||b - A x|| within 4x the FP64 rounding floor (or
    below the 1e-9 tolerance), and the mean over the steps within 1.5x of
    the FP64 path's mean (the FP64 solve's end residual, set by its
    recursive test, varies by a few rounding floors from step to step)."""
    _cuda()
    from mps_b200 import _lib
    from mps_b200.session import start
    wl = W.dambreak("c1", l0=0.02, seed=8)
    cfg = wl.config()
    h64 = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    h32 = h64.copy()
    a = start(cfg, 3, h64)
    b = start(cfg, 3, h32, precision=_lib.PREC_MIXED)
    tra, trb = [], []
    for _ in range(steps):
        a.step(1)
        b.step(1)
        ma, mb = a.metrics(), b.metrics()
        assert mb["ppe_outer"] >= 1 and mb["converged"] == 1
        assert mb["ppe_true_residual"] <= max(cfg.cg_tolerance, 4.0 * mb["ppe_rounding_floor"])
        assert ma["ppe_true_residual"] > 0.0 and ma["ppe_rounding_floor"] > 0.0
        tra.append(ma["ppe_true_residual"])
        trb.append(mb["ppe_true_residual"])
    ga, gb = a.download(), b.download()
    a.close()
    b.close()
    assert np.array_equal(ga["type"], gb["type"])
    assert _rel(gb["pressure"], ga["pressure"]) < 1e-4
    assert _rel(gb["pos"], ga["pos"]) < 1e-6
    assert np.mean(trb) <= max(cfg.cg_tolerance, 1.5 * np.mean(tra))


def test_set_precision_switches_the_form():
    """mps_set_precision: a session created FP64 and switched to the mixed
    form steps bit for bit like one created mixed; switched back, its next
    solve is the FP64 one (its pressures leave the mixed run's bits but stay
    within the mixed form's tolerance); an unknown form is rejected."""
    _cuda()
    from mps_b200 import _lib
    from mps_b200.session import start
    wl = W.dambreak("c1", l0=0.02, seed=8)
    cfg = wl.config()
    h = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    a = start(cfg, 3, h.copy())
    b = start(cfg, 3, h.copy(), precision=_lib.PREC_MIXED)
    a.set_precision(_lib.PREC_MIXED)
    with pytest.raises(_lib.MpsError) as e:
        a.set_precision(7)
    assert e.value.code == -1
    a.step(2)
    b.step(2)
    ga, gb = a.download(), b.download()
    for f in ("pos", "vel", "pressure", "n", "type", "on_surface"):
        assert np.array_equal(ga[f], gb[f]), f
    a.set_precision(_lib.PREC_FP64)
    a.step(1)
    b.step(1)
    ga, gb = a.download(), b.download()
    a.close()
    b.close()
    assert not np.array_equal(ga["pressure"], gb["pressure"])
    assert _rel(ga["pressure"], gb["pressure"]) < 1e-6


_PDL_SCRIPT = r"""
import sys
import numpy as np
from mps_b200 import types as T, workloads as W, _lib
from mps_b200.session import start
wl = W.dambreak("c1", l0=0.02, seed=9)
h = T.HostParticles(3, wl.pos, wl.vel, wl.types)
out = {}
for name, prec in (("fp64", _lib.PREC_FP64), ("mixed", _lib.PREC_MIXED)):
    hp = h.copy()
    s = start(wl.config(), 3, hp, precision=prec)
    s.step(3)
    g = s.download()
    out[name + "_p"] = g["pressure"].copy()
    out[name + "_x"] = g["pos"].copy()
    out[name + "_it"] = np.array([s.metrics()["total_iterations"]])
    s.close()
np.savez(sys.argv[1], **out)
"""


def test_programmatic_launch_is_bit_identical(tmp_path):
    """The CG loop's programmatic dependent launches change no bit: three
    steps with them (the default) and with MPS_PDL=0 give identical
    pressures, positions and iteration counts, FP64 and mixed."""
    _cuda()
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for flag in ("1", "0"):
        f = tmp_path / f"pdl{flag}.npz"
        env = dict(os.environ, MPS_PDL=flag, PYTHONPATH=root)
        r = subprocess.run([sys.executable, "-c", _PDL_SCRIPT, str(f)], cwd=root, env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        res[flag] = np.load(f)
    for k in res["1"].files:
        assert np.array_equal(res["1"][k], res["0"][k]), k
