"""Differentiation form (mps_step_adjoint, mps_b200.adjoint.Rollout) on the GPU.

Checks, with the step's discrete decisions held fixed on the forward run's
branch:
  * checkpoints: load + step reproduces the saved run bit for bit;
  * the adjoint of a few steps against a dense FP64 autograd of the same
    steps (oracle/torch_step.py, itself pinned to the C oracle's forward and
    to its own finite differences in tests/test_torch_step.py): gradients
    with respect to the initial velocities and positions, the gravity scale
    and the viscosity within 1e-6 relative L2, in 2-D and 3-D, with and
    without collision impulses;
  * against central finite differences of the GPU forward (h = 1e-6,
    agreement within 2e-4);
  * checkpoint-every-k recomputation gives the same gradient bit for bit as
    saving every step;
  * the mixed-precision forward gives the FP64 gradient within 1e-5.
"""
import numpy as np
import pytest
import torch

from mps_b200 import _lib
from mps_b200 import workloads as W

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-6
FD_TOL = 2e-4


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _case(dim: int, collide: bool, seed: int = 11):
    if dim == 2:
        wl = W.small_dambreak2d(l0=0.02, seed=seed, jitter=0.3 if collide else 0.01)
    else:
        wl = W.small_dambreak3d(seed=seed, jitter=0.45 if collide else 0.01, l0=0.025,
                                domain=(0.25, 0.2, 0.15), water=(0.1, 0.15, 0.15))
    rng = np.random.default_rng(seed)
    f = wl.types == 0
    wl.vel[f] = rng.normal(0.0, 3.0 if collide else 0.05, size=(int(f.sum()), dim))
    return wl


def _weights(n: int, dim: int, seed: int = 5, scale: float = 1.0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, dim)) * (scale / np.sqrt(n)), rng.normal(size=(n, dim)) * (scale / np.sqrt(n))


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _gpu_grad(wl, steps, every=1, precision=_lib.PREC_FP64, gscale=1.0, scale=1.0):
    from mps_b200.adjoint import Rollout
    roll = Rollout(wl.config(), wl.dim, wl.pos, wl.types, steps, every, precision=precision)
    x, u, t = roll.forward(wl.vel, gscale, roll.cfg.viscosity)
    cx, cu = _weights(wl.n, wl.dim, scale=scale)
    fl = (t == 0)[:, None]
    loss = float(np.sum(cx * x * fl) + np.sum(cu * u * fl))
    dx0, du0, dgs, dnu, _, _ = roll.backward(cx * fl, cu * fl)
    out = dict(loss=loss, dx0=dx0, du0=du0, dgs=dgs, dnu=dnu, n0=roll.n0, lam=roll.lam, types=t, x=x)
    roll.close()
    return out


def _torch_grad(wl, steps, n0, lam, scale=1.0):
    from oracle import torch_step as TS
    cfg = wl.config()
    c = TS.consts(cfg, wl.dim, n0, lam)
    x0 = torch.tensor(wl.pos, dtype=torch.float64, requires_grad=True)
    u0 = torch.tensor(wl.vel, dtype=torch.float64, requires_grad=True)
    gs = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    nu = torch.tensor(cfg.viscosity, dtype=torch.float64, requires_grad=True)
    g = torch.tensor([cfg.gravity[d] for d in range(wl.dim)], dtype=torch.float64) * gs
    x, u, key, ty = x0, u0, x0.detach().clone(), torch.tensor(wl.types, dtype=torch.int64)
    for _ in range(steps):
        x, u, key, ty, _ = TS.step(x, u, key, ty, g, nu, c)
    cx, cu = _weights(wl.n, wl.dim, scale=scale)
    fl = (ty == 0)[:, None].to(torch.float64)
    loss = torch.sum(torch.tensor(cx) * x * fl) + torch.sum(torch.tensor(cu) * u * fl)
    dx0, du0, dgs, dnu = torch.autograd.grad(loss, (x0, u0, gs, nu))
    return dict(loss=loss.item(), dx0=dx0.numpy(), du0=du0.numpy(), dgs=float(dgs), dnu=float(dnu),
                types=ty.numpy(), x=x.detach().numpy())


def test_checkpoint_roundtrip_bitexact():
    """state_save, 3 steps; state_load, 3 steps: identical particles."""
    _cuda()
    from mps_b200.session import start
    from mps_b200 import types as T
    wl = _case(3, collide=True)
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    s = start(wl.config(), 3, hp)
    s.step(2)
    buf = torch.empty(s.state_bytes(), dtype=torch.uint8, device="cuda")
    s.state_save(buf.data_ptr())
    s.step(3)
    a = s.download().copy()
    host = np.zeros(s.state_bytes(), dtype=np.uint8)
    s.state_load(buf.data_ptr())
    s.state_save(host.ctypes.data)       # host buffers work too
    s.step(3)
    b = s.download().copy()
    s.state_load(host.ctypes.data)
    s.step(3)
    c = s.download().copy()
    s.close()
    for f in ("pos", "vel", "pressure", "type", "on_surface"):
        assert np.array_equal(a[f], b[f]), f
        assert np.array_equal(a[f], c[f]), f


@pytest.mark.parametrize("dim,collide", [(2, False), (2, True), (3, False), (3, True)],
                         ids=["2d", "2d-collide", "3d", "3d-collide"])
def test_adjoint_matches_dense_autograd(dim, collide):
    _cuda()
    wl = _case(dim, collide)
    steps = 3
    gp = _gpu_grad(wl, steps)
    tr = _torch_grad(wl, steps, gp["n0"], gp["lam"])
    assert np.array_equal(gp["types"], tr["types"])
    assert _rel(gp["x"], tr["x"]) < 1e-12
    assert abs(gp["loss"] - tr["loss"]) <= 1e-10 * max(1.0, abs(tr["loss"]))
    f = wl.types == 0
    assert _rel(gp["du0"][f], tr["du0"][f]) < GRAD_TOL
    assert _rel(gp["dx0"][f], tr["dx0"][f]) < GRAD_TOL
    assert abs(gp["dgs"] - tr["dgs"]) <= GRAD_TOL * abs(tr["dgs"])
    assert abs(gp["dnu"] - tr["dnu"]) <= GRAD_TOL * abs(tr["dnu"])


def test_adjoint_independent_of_loss_scale():
    """A loss 1e-9 times smaller (its adjoint PPE right-hand side ~1e-20)
    gives the same relative gradient: the adjoint solve is normalised, so
    the CG's absolute breakdown guards cannot end it early."""
    _cuda()
    wl = _case(2, collide=False, seed=16)
    gp = _gpu_grad(wl, 3, scale=1e-9)
    tr = _torch_grad(wl, 3, gp["n0"], gp["lam"], scale=1e-9)
    f = wl.types == 0
    assert _rel(gp["du0"][f], tr["du0"][f]) < GRAD_TOL
    assert abs(gp["dgs"] - tr["dgs"]) <= GRAD_TOL * abs(tr["dgs"])


def test_adjoint_matches_central_differences():
    """Gravity scale, viscosity and three initial-velocity components of a
    2-D case (5 steps), h = 1e-6."""
    _cuda()
    from mps_b200.adjoint import Rollout
    wl = _case(2, collide=False, seed=12)
    steps = 5
    roll = Rollout(wl.config(), 2, wl.pos, wl.types, steps, every=5)
    cx, cu = _weights(wl.n, 2, seed=6)
    nu0 = roll.cfg.viscosity

    def loss(u0, gs, nu):
        x, u, t = roll.forward(u0, gs, nu)
        fl = (t == 0)[:, None]
        return float(np.sum(cx * x * fl) + np.sum(cu * u * fl)), t

    base, t0 = loss(wl.vel, 1.0, nu0)
    fl = (t0 == 0)[:, None]
    _, du0, dgs, dnu, _, _ = roll.backward(cx * fl, cu * fl)
    h = 1e-6
    lp, tp = loss(wl.vel, 1.0 + h, nu0)
    lm, tm = loss(wl.vel, 1.0 - h, nu0)
    assert np.array_equal(tp, t0) and np.array_equal(tm, t0)
    assert abs((lp - lm) / (2 * h) - dgs) <= FD_TOL * abs(dgs)
    # viscosity: h = 1e-6 absolute (nu = 1e-6 enters the step linearly); a
    # relative step of 1e-12 would sit at the ICCG stopping noise of the loss
    lp, _ = loss(wl.vel, 1.0, nu0 + h)
    lm, _ = loss(wl.vel, 1.0, nu0 - h)
    assert abs((lp - lm) / (2 * h) - dnu) <= FD_TOL * abs(dnu)
    fluid = np.nonzero(wl.types == 0)[0]
    for q in (fluid[0], fluid[len(fluid) // 2], fluid[-1]):
        for d in range(2):
            up, um = wl.vel.copy(), wl.vel.copy()
            up[q, d] += h
            um[q, d] -= h
            fd = (loss(up, 1.0, nu0)[0] - loss(um, 1.0, nu0)[0]) / (2 * h)
            assert abs(fd - du0[q, d]) <= FD_TOL * np.max(np.abs(du0)) + 1e-9, (q, d, fd, du0[q, d])
    roll.close()


def test_checkpoint_interval_gives_identical_gradient():
    _cuda()
    wl = _case(3, collide=True, seed=13)
    a = _gpu_grad(wl, 6, every=1)
    b = _gpu_grad(wl, 6, every=4)
    for k in ("du0", "dx0"):
        assert np.array_equal(a[k], b[k]), k
    assert a["dgs"] == b["dgs"] and a["dnu"] == b["dnu"]


def test_mixed_precision_gradient():
    _cuda()
    wl = _case(2, collide=True, seed=14)
    a = _gpu_grad(wl, 4)
    b = _gpu_grad(wl, 4, precision=_lib.PREC_MIXED)
    f = wl.types == 0
    assert np.array_equal(a["types"], b["types"])
    assert _rel(b["du0"][f], a["du0"][f]) < 1e-5
    assert abs(b["dgs"] - a["dgs"]) <= 1e-5 * abs(a["dgs"])


def test_torch_autograd_function():
    """The Rollout as a torch.autograd.Function: backward through a loss
    built in torch gives the same gradient as calling the adjoint directly."""
    _cuda()
    from mps_b200.adjoint import Rollout
    wl = _case(2, collide=False, seed=15)
    roll = Rollout(wl.config(), 2, wl.pos, wl.types, 4, every=2)
    u0 = torch.tensor(wl.vel, dtype=torch.float64, requires_grad=True)
    gs = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    nu = torch.tensor(roll.cfg.viscosity, dtype=torch.float64, requires_grad=True)
    x, u = roll(u0, gs, nu)
    fl = torch.tensor(wl.types == 0)[:, None]
    target = torch.tensor(wl.pos) + 0.001
    loss = torch.mean(torch.sum((x - target) ** 2, dim=1)[fl[:, 0]])
    loss.backward()
    lam = (2.0 * (x.detach() - target) / int(fl.sum())) * fl
    roll.forward(wl.vel, 1.0, roll.cfg.viscosity)
    _, du0, dgs, dnu, _, _ = roll.backward(lam.numpy(), np.zeros_like(wl.vel))
    assert np.allclose(u0.grad.numpy(), du0, rtol=0, atol=1e-14 * max(1.0, np.abs(du0).max()))
    assert float(gs.grad) == pytest.approx(dgs, rel=1e-13)
    assert float(nu.grad) == pytest.approx(dnu, rel=1e-13)
    roll.close()


# ---- driven walls ---------------------------------------------------------------

def _slosh(seed=21):
    wl = W.sloshing3d(l0=0.02, seed=seed, amp=0.01, freq=5.0, domain=(0.2, 0.15, 0.1), depth=0.08)
    rng = np.random.default_rng(seed)
    f = wl.types == 0
    wl.vel[f] = rng.normal(0.0, 0.05, size=(int(f.sum()), 3))
    return wl


def test_driven_walls_forward_matches_oracle():
    """Three driven steps against oracle_step_driven: wall positions and
    velocities bit for bit, neighbour-dependent results within the PPE
    tolerances of the undriven parity tests; amplitude 0 is the undriven step."""
    _cuda()
    from mps_b200 import config as CF
    from mps_b200 import types as T
    from mps_b200.session import start
    from oracle.pyoracle import Oracle
    wl = _slosh()
    amp, freq, axis = wl.drive
    cfg = wl.config()
    orc = Oracle(3)
    hr = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    orc.initial_params(hr, cfg)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hr.n, cfg.max_neighbors)
    cl = orc.cell_list(hr.n, re, cfg)
    assert orc.search(nl, hr, cl, re) == 0
    rest = np.ascontiguousarray(wl.pos[:, axis])
    hm = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    s = start(cfg, 3, hm)
    s.set_wall_drive(amp, freq, axis)
    for k in range(3):
        assert orc.step_driven(hr, nl, cl, cfg, rest, amp, freq, axis, k) == 0
        s.step(1)
    g, v = s.download(), hr.view
    w = (wl.types == 1) | (wl.types == 3)
    assert np.array_equal(g["pos"][w], v["pos"][w]) and np.array_equal(g["vel"][w], v["vel"][w])
    assert np.array_equal(g["type"], v["type"])
    assert _rel(g["pressure"], v["pressure"]) < 1e-8
    assert _rel(g["pos"], v["pos"]) < 1e-13
    s.close()
    # amplitude 0: the reference's fixed walls, bit for bit
    a = start(cfg, 3, T.HostParticles(3, wl.pos, wl.vel, wl.types))
    b = start(cfg, 3, T.HostParticles(3, wl.pos, wl.vel, wl.types))
    b.set_wall_drive(0.0, freq, axis)
    a.step(3)
    b.step(3)
    ga, gb = a.download(), b.download()
    for f in ("pos", "vel", "pressure"):
        assert np.array_equal(ga[f], gb[f]), f
    a.close()
    b.close()


def _torch_drive_grad(wl, steps, n0, lam):
    from oracle import torch_step as TS
    cfg = wl.config()
    amp0, freq0, axis = wl.drive
    c = TS.consts(cfg, 3, n0, lam)
    u0 = torch.tensor(wl.vel, dtype=torch.float64, requires_grad=True)
    A = torch.tensor(amp0, dtype=torch.float64, requires_grad=True)
    F = torch.tensor(freq0, dtype=torch.float64, requires_grad=True)
    g = torch.tensor([cfg.gravity[d] for d in range(3)], dtype=torch.float64)
    nu = torch.tensor(cfg.viscosity, dtype=torch.float64)
    x = torch.tensor(wl.pos, dtype=torch.float64)
    rest = x.clone()
    u, key, ty = u0, x.clone(), torch.tensor(wl.types, dtype=torch.int64)
    for k in range(steps):
        drv = dict(amp=A, freq=F, axis=axis, rest=rest, t1=float(k + 1) * cfg.dt)
        x, u, key, ty, _ = TS.step(x, u, key, ty, g, nu, c, drive=drv)
    cx, cu = _weights(wl.n, 3)
    fl = (ty == 0)[:, None].to(torch.float64)
    loss = torch.sum(torch.tensor(cx) * x * fl) + torch.sum(torch.tensor(cu) * u * fl)
    du0, dA, dF = torch.autograd.grad(loss, (u0, A, F))
    return du0.numpy(), float(dA), float(dF)


def test_adjoint_drive_gradient():
    """Gradients with respect to the drive's amplitude and frequency and the
    initial velocities: against the dense FP64 autograd (1e-6) and central
    differences of the GPU forward (h = 1e-6, 2e-4)."""
    _cuda()
    from mps_b200.adjoint import Rollout
    wl = _slosh(seed=22)
    amp, freq, axis = wl.drive
    steps = 4
    roll = Rollout(wl.config(), 3, wl.pos, wl.types, steps, every=2, drive_axis=axis)
    cx, cu = _weights(wl.n, 3)

    def loss(a, f):
        x, u, t = roll.forward(wl.vel, 1.0, roll.cfg.viscosity, a, f)
        fl = (t == 0)[:, None]
        return float(np.sum(cx * x * fl) + np.sum(cu * u * fl)), fl

    _, fl = loss(amp, freq)
    _, du0, _, _, dA, dF = roll.backward(cx * fl, cu * fl)
    tdu0, tdA, tdF = _torch_drive_grad(wl, steps, roll.n0, roll.lam)
    f = wl.types == 0
    assert _rel(du0[f], tdu0[f]) < GRAD_TOL
    assert abs(dA - tdA) <= GRAD_TOL * abs(tdA)
    assert abs(dF - tdF) <= GRAD_TOL * abs(tdF)
    h = 1e-6
    fd = (loss(amp + h, freq)[0] - loss(amp - h, freq)[0]) / (2 * h)
    assert abs(fd - dA) <= FD_TOL * abs(dA)
    fd = (loss(amp, freq + h)[0] - loss(amp, freq - h)[0]) / (2 * h)
    assert abs(fd - dF) <= FD_TOL * abs(dF)
    roll.close()


def test_adjoint_probe_pressure_loss():
    """A loss on the pressures of every step, the sloshing case's time-mean
    squared wall-probe pressure (mean over the first wall layer behind the
    +x wall below y = 0.06 m), through the probe series of Rollout and
    mps_adjoint_pressure_seed: the loss and its gradients with respect to
    the drive's amplitude and frequency, the gravity scale and the initial
    velocities against the dense FP64 autograd of the same driven steps
    (loss 1e-6, gradients 1e-6 relative)."""
    _cuda()
    from mps_b200.adjoint import Rollout
    from oracle import torch_step as TS
    wl = _slosh(seed=23)
    amp, freq, axis = wl.drive
    cfg = wl.config()
    l0, lx = cfg.particle_distance, cfg.domain_max[0]
    probe = (wl.types == 1) & (wl.pos[:, 0] > lx) & (wl.pos[:, 0] < lx + 1.5 * l0) & (wl.pos[:, 1] < 0.06)
    assert probe.sum() >= 4
    steps = 4
    roll = Rollout(cfg, 3, wl.pos, wl.types, steps, every=2, drive_axis=axis, probe=probe)
    roll.forward(wl.vel, 1.0, cfg.viscosity, amp, freq)
    ser = roll.series.copy()
    assert ser.shape == (steps,) and np.any(ser != 0.0)
    L = float(np.mean(ser ** 2))
    zero = np.zeros((wl.n, 3))
    _, du0, dgs, _, dA, dF = roll.backward(zero, zero, 2.0 * ser / steps)
    roll.close()
    # the same loss by dense autograd
    c = TS.consts(cfg, 3, roll.n0, roll.lam)
    f64 = dict(dtype=torch.float64)
    u0 = torch.tensor(wl.vel, requires_grad=True, **f64)
    A = torch.tensor(amp, requires_grad=True, **f64)
    F = torch.tensor(freq, requires_grad=True, **f64)
    gs = torch.tensor(1.0, requires_grad=True, **f64)
    g = torch.tensor([cfg.gravity[d] for d in range(3)], **f64) * gs
    nu = torch.tensor(cfg.viscosity, **f64)
    x = torch.tensor(wl.pos, **f64)
    rest = x.clone()
    u, key, ty = u0, x.clone(), torch.tensor(wl.types, dtype=torch.int64)
    pidx = torch.tensor(np.flatnonzero(probe))
    tl = torch.zeros((), **f64)
    for k in range(steps):
        drv = dict(amp=A, freq=F, axis=axis, rest=rest, t1=float(k + 1) * cfg.dt)
        x, u, key, ty, info = TS.step(x, u, key, ty, g, nu, c, drive=drv)
        tl = tl + info["P"][pidx].mean() ** 2
    tl = tl / steps
    tdu0, tdA, tdF, tdgs = torch.autograd.grad(tl, (u0, A, F, gs))
    assert abs(L - tl.item()) <= 1e-6 * abs(tl.item())
    f = wl.types == 0
    assert _rel(du0[f], tdu0.numpy()[f]) < GRAD_TOL
    assert abs(dA - float(tdA)) <= GRAD_TOL * abs(float(tdA))
    assert abs(dF - float(tdF)) <= GRAD_TOL * abs(float(tdF))
    assert abs(dgs - float(tdgs)) <= GRAD_TOL * abs(float(tdgs))


def test_config3_geometry_fd_50_steps():
    """The config-3 set-up at full size (2-D dam break, l0 = 0.005, 6,788
    particles): 50 steps from rest, loss = mean squared distance of the fluid
    to a target run with gravity x 1.05 and Gaussian initial velocities
    (sigma 0.05 m/s), checkpoints every 10.  dL/d(gravity scale) from the
    adjoint against central differences (h = 1e-6, 1e-5 relative), with no
    surface flag differing between the base and the +-h runs (a flip would
    be a discontinuity, which the adjoint holds fixed).  The viscosity's
    finite difference is covered by the small case: here the loss barely
    depends on it and h = 1e-6 would double it."""
    _cuda()
    from mps_b200.adjoint import Rollout
    wl = W.dambreak("c3")
    cfg = wl.config()
    steps = 50
    rng = np.random.default_rng(7)
    f0 = wl.types == 0
    vt = np.zeros_like(wl.vel)
    vt[f0] = rng.normal(0.0, 0.05, size=(int(f0.sum()), 2))
    roll = Rollout(cfg, 2, wl.pos, wl.types, steps, every=10)
    xt, _, tt = roll.forward(vt, 1.05, cfg.viscosity)
    u0 = np.zeros_like(wl.vel)

    def run(gs, nu):
        roll._set_params(gs, nu)
        roll._upload(u0)
        roll.sess.set_initial_params(roll.n0, roll.lam, roll.n0_count)
        roll.sess.neighbor_search()
        roll.ckpts, flags = [], []
        for s in range(steps):
            if s % roll.every == 0:
                roll.ckpts.append(roll._save())
            roll.sess.step(1)
            flags.append(roll.sess.download()["on_surface"].copy())
        x, u, t = roll._final()
        m = (t == 0) & (tt == 0)
        d = (x - xt)[m]
        return float(np.mean(np.sum(d * d, axis=1))), x, m, np.array(flags)

    _, x, m, fb = run(1.0, cfg.viscosity)
    lam = np.zeros_like(x)
    lam[m] = 2.0 * (x - xt)[m] / m.sum()
    _, _, dgs, _, _, _ = roll.backward(lam, np.zeros_like(x))
    h = 1e-6
    lp, _, _, fp = run(1.0 + h, cfg.viscosity)
    lm, _, _, fm = run(1.0 - h, cfg.viscosity)
    assert np.array_equal(fp, fb) and np.array_equal(fm, fb)
    assert abs((lp - lm) / (2 * h) - dgs) <= 1e-5 * abs(dgs)
    roll.close()
