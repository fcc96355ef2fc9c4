"""The IC(0) preconditioner of the GPU solver pinned against the oracle.

The solver numbers the PPE unknowns in block colour order (cells as blocks,
2^dim colours) and factors that permuted matrix with the reference's IC(0)
(pressure_solver.c:156-232); oracle_ic0_csr restates the reference
algorithm on any numbering.  Checked through the C ABI, after one step:

  * the factor F (L below the diagonal, 1/L_ii on it, L^T above) against
    the oracle's factor of the same matrix: relative L2 <= 1e-13, every
    entry within 1e-10 relative (the GPU sums each entry's sparse dot product
    across a warp, the oracle in ascending order);
  * the in-cell block inverses (k_cell_inverse) against the oracle's
    substitution from the same factor: relative L2 <= 1e-13;
  * one application z = (L L^T)^-1 r of the device sweeps (the persistent
    ICCG kernel's apply mode and both launch-per-colour sweep kernels)
    against the oracle's triangular solves: relative L2 <= 1e-11 in FP64,
    <= 1e-4 with the mixed form's FP32 copy of the factor.

Cases: a 3-D and a 2-D dam break, and a densely packed 3-D column (cells of
up to ~90 unknowns) that reaches the sweeps' unstaged (41-64 unknowns) and
substitution (> 64) paths.
"""
import numpy as np
import pytest

from mps_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


CASES = {
    "dambreak3d": lambda: W.dambreak("c1", l0=0.02, seed=3),
    "dambreak2d": lambda: W.small_dambreak2d(l0=0.01, seed=4),
    "dense3d": lambda: W.small_dambreak3d(l0=0.014, seed=5, influence_ratio_lap="4.43"),
}


def _stepped(name, precision=0, monkeypatch=None, sweep="1"):
    from mps_b200 import types as T
    from mps_b200.session import start
    if monkeypatch is not None:
        monkeypatch.setenv("MPS_SWEEP", sweep)
    wl = CASES[name]()
    hp = T.HostParticles(wl.dim, wl.pos, wl.vel, wl.types)
    s = start(wl.config(), wl.dim, hp, precision=precision)
    s.step(1)
    return s


@pytest.mark.parametrize("name", sorted(CASES))
def test_factor_and_block_inverses_match_the_oracle(name, oracle3):
    _cuda()
    s = _stepped(name)
    try:
        f = s.ic0()
        cells, off, inv, crow = s.cell_blocks()
    finally:
        s.close()
    rp, ci, A, F = f["row_ptr"], f["col"], f["A"], f["F"]
    n_eq = len(rp) - 1
    assert n_eq > 0 and crow[0] == 0 and crow[-1] == n_eq
    # rows cell by cell, colour by colour
    assert np.array_equal(np.cumsum(cells[:, 1])[:-1], cells[1:, 0] - cells[0, 0])
    Fo = oracle3.ic0_csr(rp, ci, A)
    assert np.all(np.isfinite(F))
    assert _rel(F, Fo) <= 1e-13, _rel(F, Fo)
    big = np.abs(Fo) > 0
    assert np.max(np.abs(F[big] - Fo[big]) / np.abs(Fo[big])) <= 1e-10
    # diagonal slots hold 1 / L_ii > 0
    rows = np.repeat(np.arange(n_eq), np.diff(rp))
    assert np.all(F[ci == rows] > 0)
    io = oracle3.cell_inverses(cells, off, rp, ci, F)
    m = cells[:, 1]
    assert np.count_nonzero(m <= 64) > 0
    assert _rel(inv[: off[-1]], io[: off[-1]]) <= 1e-13, _rel(inv[: off[-1]], io[: off[-1]])
    if name == "dense3d":
        assert m.max() > 64 and np.count_nonzero((m > 40) & (m <= 64)) > 0, m.max()


@pytest.mark.parametrize("sweep", ["2", "1", "0"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_preconditioner_apply_matches_the_oracle(name, sweep, oracle3, monkeypatch):
    _cuda()
    s = _stepped(name, monkeypatch=monkeypatch, sweep=sweep)
    try:
        f = s.ic0()
        r = np.random.default_rng(7).normal(size=len(f["b"]))
        z = s.apply_preconditioner(r)
        z2 = s.apply_preconditioner(f["b"])
    finally:
        s.close()
    zo = oracle3.ic0_apply_csr(f["row_ptr"], f["col"], f["F"], r)
    assert _rel(z, zo) <= 1e-11, _rel(z, zo)
    zo2 = oracle3.ic0_apply_csr(f["row_ptr"], f["col"], f["F"], f["b"])
    assert _rel(z2, zo2) <= 1e-11, _rel(z2, zo2)


@pytest.mark.parametrize("name", ["dambreak3d", "dense3d"])
def test_mixed_form_preconditioner_is_the_fp32_factor(name, oracle3):
    """After a mixed-form step the sweeps use the FP32 copy of the factor:
    the apply agrees with the FP64 oracle to FP32 accuracy, not better."""
    _cuda()
    s = _stepped(name, precision=1)
    try:
        f = s.ic0()
        r = np.random.default_rng(8).normal(size=len(f["b"]))
        z = s.apply_preconditioner(r)
    finally:
        s.close()
    zo = oracle3.ic0_apply_csr(f["row_ptr"], f["col"], f["F"], r)
    e = _rel(z, zo)
    assert 1e-12 < e <= 1e-4, e
