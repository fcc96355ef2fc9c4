"""CPU checks of the torch.autograd plumbing of mps_b200.adjoint.Rollout
(no GPU: a stand-in object with Rollout's forward/backward contract takes the
place of the session-backed rollout).  With a probe, calling the rollout
returns (x_T, u_T, probe series) and the series' gradient reaches backward
as lam_series; without one it returns (x_T, u_T) and backward gets no
series adjoint; the returned gradients land on the inputs."""
import numpy as np
import pytest
import torch

from mps_b200.adjoint import Rollout


class _Stand:
    __call__ = Rollout.__call__

    def __init__(self, n=5, dim=3, steps=4, probe=True):
        self.n, self.dim, self.steps = n, dim, steps
        self.probe = np.array([1, 3]) if probe else None
        self.series = np.zeros(0)
        self.calls = []

    def forward(self, u0, gs, nu, amp, freq):
        self.calls.append(("forward", gs, nu, amp, freq))
        x = np.arange(self.n * self.dim, dtype=np.float64).reshape(self.n, self.dim) * gs
        u = u0 + nu
        self.series = np.linspace(1.0, 2.0, self.steps) * amp if self.probe is not None else np.zeros(0)
        return x, u, np.zeros(self.n, dtype=np.int32)

    def backward(self, lam_x, lam_u, lam_series=None):
        self.calls.append(("backward", lam_x.copy(), lam_u.copy(), None if lam_series is None else lam_series.copy()))
        du0 = np.full((self.n, self.dim), 0.5)
        return np.zeros((self.n, self.dim)), du0, 2.0, 3.0, 4.0, 5.0


def _inputs(n=5, dim=3):
    f64 = dict(dtype=torch.float64)
    return (torch.zeros((n, dim), requires_grad=True, **f64), torch.tensor(1.5, requires_grad=True, **f64),
            torch.tensor(1e-6, requires_grad=True, **f64), torch.tensor(0.01, requires_grad=True, **f64),
            torch.tensor(1.5, requires_grad=True, **f64))


def test_probe_series_gradient_reaches_backward():
    roll = _Stand(probe=True)
    u0, gs, nu, amp, freq = _inputs()
    out = roll(u0, gs, nu, amp, freq)
    assert len(out) == 3
    x, u, series = out
    assert series.shape == (roll.steps,)
    loss = (series ** 2).mean() + x.sum()
    loss.backward()
    kind, lx, lu, ls = roll.calls[-1]
    assert kind == "backward"
    assert np.array_equal(lx, np.ones((roll.n, roll.dim)))
    assert np.array_equal(lu, np.zeros((roll.n, roll.dim)))
    expect = 2.0 * series.detach().numpy() / roll.steps
    assert ls is not None and np.allclose(ls, expect, rtol=0, atol=1e-15)
    assert torch.equal(u0.grad, torch.full((roll.n, roll.dim), 0.5, dtype=torch.float64))
    assert (gs.grad.item(), nu.grad.item(), amp.grad.item(), freq.grad.item()) == (2.0, 3.0, 4.0, 5.0)


def test_without_probe_two_outputs_and_no_series_adjoint():
    roll = _Stand(probe=False)
    u0, gs, nu, amp, freq = _inputs()
    out = roll(u0, gs, nu, amp, freq)
    assert len(out) == 2
    x, u = out
    (u.sum() * 2.0).backward()
    kind, lx, lu, ls = roll.calls[-1]
    assert ls is None
    assert np.array_equal(lu, np.full((roll.n, roll.dim), 2.0))
    assert np.array_equal(lx, np.zeros((roll.n, roll.dim)))
    assert u0.grad is not None


def test_backward_rejects_series_without_probe():
    """Rollout.backward refuses a series adjoint when it recorded no series."""
    r = Rollout.__new__(Rollout)
    r.probe = None
    with pytest.raises(ValueError):
        Rollout.backward(r, np.zeros((2, 3)), np.zeros((2, 3)), np.zeros(4))


@pytest.mark.parametrize("probe,msg", [([], "selects no particle"), ([0, 10 ** 9], "out of range"),
                                       ([-1], "out of range"), (np.zeros(3, dtype=bool), "one entry per particle")])
def test_probe_validated_before_any_gpu_work(probe, msg):
    """A bad probe is rejected by the constructor before a session exists."""
    from mps_b200 import workloads as W
    wl = W.small_dambreak2d(l0=0.05, seed=1)
    with pytest.raises(ValueError, match=msg):
        Rollout(wl.config(), 2, wl.pos, wl.types, steps=2, probe=np.asarray(probe))
