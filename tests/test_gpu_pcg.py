"""The persistent ICCG kernel (k_pcg, one cooperative launch per batch of
CG iterations) against the launch-per-colour form of the same solve.

Both solve the step's PPE with the block-colour IC(0) preconditioner of
pressure_solver.c:156-322 and stop on the reference's test sqrt(r.r) < 1e-9
(pressure_solver.c:290), so they agree to the solve's round-off; the
persistent kernel sums in another order (its own grid), so not bit for bit.
Checked through the C ABI:

  * one and five FP64 steps (3-D), one 2-D step and a mixed-form step:
    pressures within 1e-8 relative L2 of the launch-per-colour form,
    positions within 1e-12, the same surface flags and types; iteration
    counts within 3 % in 3-D (the small 2-D case ends its solve where the
    recursive residual creeps along the tolerance, so there 10 %);
  * two runs of the persistent kernel are bit-identical (fixed-order grid
    sums, same grid);
  * the mixed form's FP32 matrix and cross runs read as packed (value,
    column) words (MPS_PACK=1, the default) or as separate arrays
    (MPS_PACK=0): the same sums in the same order, so bit-identical
    pressures, positions and iteration counts over three steps, on the
    dam break and on a densely packed column (unstaged and substituted
    cells);
  * the grid barrier's bounded wait: with the poll limit lowered to zero
    (MPS_TEST_BAR_POLLS=0) the barrier gives up at once, the kernel returns
    and the step fails with MPS_ERR_CUDA; the device stays usable and a
    fresh session then steps normally.
"""
import numpy as np
import pytest

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


def _run(monkeypatch, sweep, wl, steps, precision=0, pack="1"):
    from mps_b200.session import start
    monkeypatch.setenv("MPS_SWEEP", sweep)
    monkeypatch.setenv("MPS_PACK", pack)
    hp = T.HostParticles(wl.dim, wl.pos, wl.vel, wl.types)
    s = start(wl.config(), wl.dim, hp, precision=precision)
    its = []
    try:
        for _ in range(steps):
            s.step(1)
            its.append(s.metrics()["ppe_iterations"])
        g = s.download()
    finally:
        s.close()
    return g, np.array(its)


@pytest.mark.parametrize("case", ["3d-1", "3d-5", "2d-1", "3d-mixed"])
def test_persistent_pcg_matches_launch_per_colour(case, monkeypatch):
    _cuda()
    if case.startswith("2d"):
        wl = W.small_dambreak2d(l0=0.01, seed=4)
    else:
        wl = W.dambreak("c1", l0=0.02, seed=3)
    steps = 5 if case == "3d-5" else 1
    prec = 1 if case == "3d-mixed" else 0
    ga, ia = _run(monkeypatch, "2", wl, steps, prec)
    gb, ib = _run(monkeypatch, "0", wl, steps, prec)
    assert np.array_equal(ga["on_surface"], gb["on_surface"])
    assert np.array_equal(ga["type"], gb["type"])
    assert _rel(ga["pressure"], gb["pressure"]) <= 1e-8, _rel(ga["pressure"], gb["pressure"])
    assert _rel(ga["pos"], gb["pos"]) <= 1e-12
    band = 0.10 if case.startswith("2d") else 0.03
    assert np.all(np.abs(ia - ib) <= np.maximum(2, band * ib)), (ia, ib)


def test_persistent_pcg_is_deterministic(monkeypatch):
    _cuda()
    wl = W.dambreak("c1", l0=0.02, seed=6)
    ga, ia = _run(monkeypatch, "2", wl, 3)
    gb, ib = _run(monkeypatch, "2", wl, 3)
    assert np.array_equal(ia, ib)
    assert np.array_equal(ga["pressure"], gb["pressure"])
    assert np.array_equal(ga["pos"], gb["pos"])


@pytest.mark.parametrize("case", ["dambreak3d", "dense3d"])
def test_packed_fp32_entries_are_bit_identical(case, monkeypatch):
    _cuda()
    if case == "dense3d":
        wl = W.small_dambreak3d(l0=0.014, seed=5, influence_ratio_lap="4.43")
    else:
        wl = W.dambreak("c1", l0=0.02, seed=3)
    ga, ia = _run(monkeypatch, "0", wl, 3, precision=1, pack="1")
    gb, ib = _run(monkeypatch, "0", wl, 3, precision=1, pack="0")
    assert np.array_equal(ia, ib), (ia, ib)
    assert np.array_equal(ga["pressure"], gb["pressure"])
    assert np.array_equal(ga["pos"], gb["pos"])
    assert np.array_equal(ga["vel"], gb["vel"])


def test_grid_barrier_timeout_is_reported(monkeypatch):
    _cuda()
    from mps_b200 import _lib
    from mps_b200.session import start
    wl = W.dambreak("c1", l0=0.02, seed=3)
    monkeypatch.setenv("MPS_SWEEP", "2")
    monkeypatch.setenv("MPS_TEST_BAR_POLLS", "0")
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    s = start(wl.config(), 3, hp)
    try:
        with pytest.raises(_lib.MpsError) as e:
            s.step(1)
        assert e.value.code == -2   # MPS_ERR_CUDA
        assert "grid barrier" in str(e.value)
    finally:
        s.close()
    monkeypatch.delenv("MPS_TEST_BAR_POLLS")
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    s = start(wl.config(), 3, hp)
    try:
        s.step(1)
        m = s.metrics()
    finally:
        s.close()
    assert m["converged"] == 1 and m["ppe_iterations"] > 0
