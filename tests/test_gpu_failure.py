"""Failure paths of the step on the GPU, made on the host or by a bounded
wait that a test shortens; none faults or hangs the device.

  * the iteration cap: with cg_max_iter = 1 the PCG stops after one
    iteration, as the reference's loop does (pressure_solver.c:290); the
    step completes and the metrics report converged = 0, in both precision
    forms (MPS_ERR_NOT_CONVERGED is reported, never raised by default);
  * a NaN velocity in the input state: the NaN spreads through the
    viscosity sum to the particle's neighbours in this step, their
    positions become NaN and remove_out_of_bounds turns them into GHOST
    particles with P = n = v = a = 0 (boundary.c:33-61); every field equals
    the oracle's (NaN where it is NaN);
  * the bulk copy of the launch-per-colour sweep: with its first wait cut
    to zero polls (MPS_TEST_MBAR_POLLS=0) the CTA records the timeout,
    still waits for its copy under the long bound and returns; the step
    fails with MPS_ERR_CUDA and a new session on the same device steps
    normally.
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


@pytest.mark.parametrize("precision", [0, 1])
def test_iteration_cap_reports_not_converged(precision):
    _cuda()
    from mps_b200.session import start
    from oracle.pyoracle import Oracle
    wl = W.small_dambreak3d(l0=0.02, seed=31, cg_max_iter=1)
    cfg = wl.config()
    assert cfg.cg_max_iter == 1
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    s = start(cfg, 3, hp, precision=precision)
    try:
        s.step(1)
        m = s.metrics()
        g = s.download()
    finally:
        s.close()
    assert m["converged"] == 0
    assert m["ppe_iterations"] == 1
    assert np.all(np.isfinite(g["pressure"]))
    # the reference's loop stops after one iteration as well
    orc = Oracle(3)
    ho = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    orc.initial_params(ho, cfg)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(ho.n, cfg.max_neighbors)
    cl = orc.cell_list(ho.n, re, cfg)
    assert orc.search(nl, ho, cl, re) == 0
    assert orc.step(ho, nl, cl, cfg) == 0
    assert orc.lib.oracle_last_iterations() == 1


def test_nan_velocity_becomes_ghost():
    _cuda()
    from mps_b200.session import Session
    from oracle.pyoracle import Oracle
    wl = W.small_dambreak3d(l0=0.02, seed=32)
    cfg = wl.config()
    orc = Oracle(3)
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hp.n, cfg.max_neighbors)
    cl = orc.cell_list(hp.n, re, cfg)
    assert orc.search(nl, hp, cl, re) == 0
    # an interior fluid particle
    fluid = np.nonzero(hp.view["type"] == 0)[0]
    k = int(fluid[len(fluid) // 2])
    hp.view["vel"][k, 0] = np.nan
    m = cfg.max_neighbors
    hg = hp.copy()
    nb_prev, cnt_prev = nl.neighbors[: hp.n * m].copy(), nl.count[: hp.n].copy()
    assert orc.step(hp, nl, cl, cfg) == 0
    with Session(cfg, 3, hg.n) as s:
        s.upload(hg)
        s.set_initial_params(hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count)
        s.step_with_list(nb_prev, cnt_prev, m)
        g = s.download()
    o = hp.view
    ghosts = np.nonzero(o["type"] == 2)[0]
    assert k in ghosts and len(ghosts) > 1          # the particle and its viscosity neighbours
    assert np.array_equal(g["type"], o["type"])
    for f in ("pressure", "n"):
        assert np.all(g[f][ghosts] == 0.0), f
    for f in ("vel", "acc"):
        assert np.all(g[f][ghosts] == 0.0), f
    for f in ("n", "on_surface", "neighbor_count"):
        assert np.array_equal(g[f], o[f], equal_nan=True), f
    live = o["type"] != 2
    assert _rel(g["pressure"][live], o["pressure"][live]) < 1e-8
    assert _rel(g["vel"][live], o["vel"][live]) < 1e-10
    assert _rel(g["pos"][live], o["pos"][live]) < 1e-14
    assert np.array_equal(np.isnan(g["pos"]), np.isnan(o["pos"]))


def test_staged_copy_timeout_is_reported(monkeypatch):
    _cuda()
    from mps_b200.session import start
    wl = W.dambreak("c1", l0=0.02, seed=33)
    monkeypatch.setenv("MPS_SWEEP", "0")
    monkeypatch.setenv("MPS_TEST_MBAR_POLLS", "0")
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    s = start(wl.config(), 3, hp)
    try:
        with pytest.raises(Exception) as e:
            s.step(1)
        assert getattr(e.value, "code", None) == -2   # MPS_ERR_CUDA
        assert "bulk copy" in str(e.value)
    finally:
        s.close()
    monkeypatch.delenv("MPS_TEST_MBAR_POLLS")
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    s = start(wl.config(), 3, hp)
    try:
        s.step(1)
        assert s.metrics()["converged"] == 1
    finally:
        s.close()
