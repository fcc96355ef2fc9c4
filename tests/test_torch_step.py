"""Pins oracle/torch_step.py, the dense FP64 autograd restatement of the step
that checks the adjoint kernels:
  * forward: three steps agree with the C restatement (oracle_step), which
    is itself bit-identical to the reference built from source -- pressure,
    velocity and position within 1e-12 relative L2, types and surface flags
    identical -- in 2-D and 3-D, including collision impulses;
  * gradient: autograd of a few steps against central finite differences of
    the same module (h = 1e-6), for the gravity scale, the viscosity and
    initial velocities.
"""
import numpy as np
import pytest
import torch

from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W


def _case(dim, seed=3, collide=False):
    if dim == 2:
        wl = W.small_dambreak2d(l0=0.02, seed=seed, jitter=0.3 if collide else 0.01)
    else:
        wl = W.small_dambreak3d(seed=seed, jitter=0.45 if collide else 0.01, l0=0.025,
                                domain=(0.25, 0.2, 0.15), water=(0.1, 0.15, 0.15))
    if collide:
        rng = np.random.default_rng(seed)
        f = wl.types == 0
        wl.vel[f] = rng.normal(0.0, 3.0, size=(int(f.sum()), dim))
    return wl


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("dim,collide", [(2, False), (2, True), (3, True)], ids=["2d", "2d-collide", "3d-collide"])
def test_torch_step_matches_oracle(dim, collide):
    from oracle import torch_step as TS
    from oracle.pyoracle import Oracle
    wl = _case(dim, collide=collide)
    cfg = wl.config()
    orc = Oracle(dim)
    hp = T.HostParticles(dim, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)
    c = TS.consts(cfg, dim, hp.ps.n0, hp.ps.lambda_)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hp.n, cfg.max_neighbors)
    cl = orc.cell_list(hp.n, re, cfg)
    assert orc.search(nl, hp, cl, re) == 0
    x = torch.tensor(wl.pos, dtype=torch.float64)
    u = torch.tensor(wl.vel, dtype=torch.float64)
    key, ty = x.clone(), torch.tensor(wl.types, dtype=torch.int64)
    g = torch.tensor([cfg.gravity[d] for d in range(dim)], dtype=torch.float64)
    nu = torch.tensor(cfg.viscosity, dtype=torch.float64)
    for _ in range(3):
        x, u, key, ty, info = TS.step(x, u, key, ty, g, nu, c)
        assert orc.step(hp, nl, cl, cfg) == 0
        v = hp.view
        assert np.array_equal(ty.numpy(), v["type"])
        assert np.array_equal(info["surf"].numpy().astype(np.int32), v["on_surface"])
        assert _rel(info["P"].numpy(), v["pressure"]) < 1e-12
        assert _rel(u.numpy(), v["vel"]) < 1e-12
        assert _rel(x.numpy(), v["pos"]) < 1e-12


def test_torch_step_gradient_matches_central_differences():
    from oracle import torch_step as TS
    from oracle.pyoracle import Oracle
    wl = _case(2, seed=4, collide=True)
    cfg = wl.config()
    hp = T.HostParticles(2, wl.pos, wl.vel, wl.types)
    Oracle(2).initial_params(hp, cfg)
    c = TS.consts(cfg, 2, hp.ps.n0, hp.ps.lambda_)
    rng = np.random.default_rng(9)
    cx = torch.tensor(rng.normal(size=(wl.n, 2)) / np.sqrt(wl.n))
    g0 = torch.tensor([cfg.gravity[0], cfg.gravity[1]], dtype=torch.float64)

    def loss(u0, gs, nu):
        x, u = torch.tensor(wl.pos), u0
        key, ty = x.clone(), torch.tensor(wl.types, dtype=torch.int64)
        for _ in range(3):
            x, u, key, ty, _ = TS.step(x, u, key, ty, g0 * gs, nu, c)
        return torch.sum(cx * x * (ty == 0)[:, None])

    u0 = torch.tensor(wl.vel, requires_grad=True)
    gs = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    nu = torch.tensor(cfg.viscosity, dtype=torch.float64, requires_grad=True)
    du0, dgs, dnu = torch.autograd.grad(loss(u0, gs, nu), (u0, gs, nu))
    h = 1e-6
    with torch.no_grad():
        u = torch.tensor(wl.vel)
        one = torch.tensor(1.0, dtype=torch.float64)
        fd = (loss(u, one + h, nu) - loss(u, one - h, nu)) / (2 * h)
        assert abs(float(fd) - float(dgs)) <= 1e-5 * abs(float(dgs))
        hn = h * cfg.viscosity
        fd = (loss(u, gs, nu + hn) - loss(u, gs, nu - hn)) / (2 * hn)
        assert abs(float(fd) - float(dnu)) <= 1e-4 * abs(float(dnu)) + 1e-9
        fluid = np.nonzero(wl.types == 0)[0]
        for q in (fluid[0], fluid[-1]):
            up, um = u.clone(), u.clone()
            up[q, 1] += h
            um[q, 1] -= h
            fd = (loss(up, gs, nu) - loss(um, gs, nu)) / (2 * h)
            assert abs(float(fd) - float(du0[q, 1])) <= 1e-5 * float(torch.max(torch.abs(du0))) + 1e-10


def test_torch_step_driven_matches_oracle():
    """Driven walls: three steps against oracle_step_driven (1e-12), and the
    drive gradients against central differences (h = 1e-6)."""
    from oracle import torch_step as TS
    from oracle.pyoracle import Oracle
    wl = W.sloshing3d(l0=0.02, seed=21, amp=0.01, freq=5.0, domain=(0.2, 0.15, 0.1), depth=0.08)
    amp, freq, axis = wl.drive
    cfg = wl.config()
    orc = Oracle(3)
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    orc.initial_params(hp, cfg)
    c = TS.consts(cfg, 3, hp.ps.n0, hp.ps.lambda_)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hp.n, cfg.max_neighbors)
    cl = orc.cell_list(hp.n, re, cfg)
    assert orc.search(nl, hp, cl, re) == 0
    rest_np = np.ascontiguousarray(wl.pos[:, axis])
    g = torch.tensor([cfg.gravity[d] for d in range(3)], dtype=torch.float64)
    nu = torch.tensor(cfg.viscosity, dtype=torch.float64)

    def run(A, F, oracle=False):
        x = torch.tensor(wl.pos, dtype=torch.float64)
        rest = x.clone()
        u, key, ty = torch.tensor(wl.vel, dtype=torch.float64), x.clone(), torch.tensor(wl.types, dtype=torch.int64)
        for k in range(3):
            drv = dict(amp=A, freq=F, axis=axis, rest=rest, t1=float(k + 1) * cfg.dt)
            x, u, key, ty, info = TS.step(x, u, key, ty, g, nu, c, drive=drv)
            if oracle:
                assert orc.step_driven(hp, nl, cl, cfg, rest_np, amp, freq, axis, k) == 0
                v = hp.view
                assert np.array_equal(ty.numpy(), v["type"])
                assert _rel(info["P"].numpy(), v["pressure"]) < 1e-12
                assert _rel(x.numpy(), v["pos"]) < 1e-12
                assert _rel(u.numpy(), v["vel"]) < 1e-12
        return x

    run(torch.tensor(amp, dtype=torch.float64), torch.tensor(freq, dtype=torch.float64), oracle=True)
    rng = np.random.default_rng(3)
    cx = torch.tensor(rng.normal(size=(wl.n, 3)))
    A = torch.tensor(amp, dtype=torch.float64, requires_grad=True)
    F = torch.tensor(freq, dtype=torch.float64, requires_grad=True)
    dA, dF = torch.autograd.grad(torch.sum(cx * run(A, F)), (A, F))
    h = 1e-6
    with torch.no_grad():
        a, f = torch.tensor(amp, dtype=torch.float64), torch.tensor(freq, dtype=torch.float64)
        fd = (torch.sum(cx * run(a + h, f)) - torch.sum(cx * run(a - h, f))) / (2 * h)
        assert abs(float(fd) - float(dA)) <= 1e-5 * abs(float(dA))
        fd = (torch.sum(cx * run(a, f + h)) - torch.sum(cx * run(a, f - h))) / (2 * h)
        assert abs(float(fd) - float(dF)) <= 1e-5 * abs(float(dF))
