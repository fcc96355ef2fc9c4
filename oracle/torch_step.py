"""Dense FP64 restatement of one MPS time step in PyTorch, differentiable by
autograd -- test infrastructure only (the checker for the adjoint kernels).

It follows the same step as the C restatement (oracle/mps_oracle.c,
``oracle_step``; reference 3P ``simulation.c:19-118``, 2D
``simulation.c:25-118``) on dense N x N pair matrices, so it is meant for
small N (a few thousand particles at most).  Every discrete decision of the
step is taken without gradient from the forward values and then held fixed:
list membership (previous step's list for viscosity and collision, fresh list
after the collision), the collision partners, their order and the
``vn > 0`` branch, the free-surface flags, the PPE unknown set, the P_min
argument and ghosting.  Everything continuous -- kernel weights, the PPE
matrix and right-hand side, the pressure solve, P_min's value, the
gradient, the integration -- carries gradients, so autograd of this module is
the FP64 reference gradient of the step with topology held
piecewise-constant.

Supported switches: those of the dam-break configurations (hs_mode 0,
ppe_type 0, cmps_gradient 0, no clamp, no surface tension); surface
detection by number density or by count.

Source lines followed (reference 3P unless noted):
  kernel weight          kernel.c:12-20
  viscosity              operators.c:50-85, simulation.c:31-43
  explicit update        simulation.c:52-67
  collision              operators.c:371-446 (3-D, list order);
                         2D operators.c:324-392 (all pairs, index order)
  neighbour search       neighbor_search.c:146-240 (membership r2 < re^2)
  number density         operators.c:17-38
  surface flags          operators.c:206-219 (count form :226-267)
  PPE                    pressure_solver.c:411-551 (matrix, rhs :328-340)
  P_min and gradient     operators.c:102-181
  correction, boundary   simulation.c:100-117, boundary.c:12-61
  driven walls           no counterpart (oracle_step_driven; fixed walls at A = 0)
"""
from __future__ import annotations

import numpy as np
import torch

FLUID, WALL, GHOST, DUMMY = 0, 1, 2, 3


def consts(cfg, dim: int, n0: float, lam: float) -> dict:
    """Scalar constants of the step from a SimConfig and n0 / lambda, with
    the reference's expressions."""
    l0 = cfg.particle_distance
    re_lap, re_n = cfg.influence_radius_lap, cfg.influence_radius_n
    re_list = max(re_lap, re_n)
    dt = cfg.dt
    m = l0 * (cfg.wall_layers + 1)
    margin = 4.0 * re_list
    origin = [cfg.domain_min[d] - margin for d in range(dim)]
    dims = [int(((cfg.domain_max[d] + margin) - origin[d]) / re_list) + 2 for d in range(dim)]
    cd = cfg.collision_distance_ratio * l0
    return dict(
        dim=dim, l0=l0, rmin=0.01 * l0, re_lap=re_lap, re_n=re_n, re_list2=re_list * re_list,
        coeff=2.0 * dim / (n0 * lam), n0=n0, density=cfg.density, dt=dt,
        rhs_k=cfg.relaxation_coeff * (cfg.density / (dt * dt)),
        neg_grad=-((float(dim)) / n0), grad_r2min=l0 * l0 * 1.0e-12,
        surf_thr=cfg.surface_threshold * n0, surf_method=cfg.surface_detection_method,
        count_thr=cfg.surface_count_threshold, re_n2=re_n * re_n,
        col_on=(cfg.collision_distance_ratio > 0.0) or dim == 2, col2=cd * cd, col_rmin=1.0e-12 * l0,
        half1pe=(1.0 + cfg.restitution_coeff) * 0.5,
        oob_lo=[cfg.domain_min[d] - m for d in range(dim)], oob_hi=[cfg.domain_max[d] + m for d in range(dim)],
        origin=origin, cs_inv=1.0 / re_list, dims=dims,
    )


def _r2(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """((0 + dx^2) + dy^2) + dz^2 with dx = b_j - a_i, for all pairs (i, j)."""
    s = torch.zeros(a.shape[0], b.shape[0], dtype=a.dtype, device=a.device)
    for d in range(a.shape[1]):
        t = b[None, :, d] - a[:, None, d]
        s = s + t * t
    return s


def _kw(r: torch.Tensor, re: float, rmin: float) -> torch.Tensor:
    return torch.where(r < re, re / torch.clamp(r, min=rmin) - 1.0, torch.zeros_like(r))


def _safe_r(r2: torch.Tensor, mask: torch.Tensor) -> torch.Tensor:
    return torch.sqrt(torch.where(mask, r2, torch.ones_like(r2)))


def _members(key: torch.Tensor, types: torch.Tensor, c: dict) -> torch.Tensor:
    act = types != GHOST
    m = (_r2(key, key) < c["re_list2"]) & act[:, None] & act[None, :]
    m.fill_diagonal_(False)
    return m


def _cell_lin(key: torch.Tensor, c: dict) -> np.ndarray:
    k = key.detach().cpu().numpy()
    lin = np.zeros(k.shape[0], dtype=np.int64)
    for d in reversed(range(c["dim"])):
        t = np.trunc((k[:, d] - c["origin"][d]) * c["cs_inv"]).astype(np.int64)
        lin = lin * c["dims"][d] + t
    return lin


def _collision(xs, us, key, types, mprev, c):
    """Sequential impulses per fluid particle (frozen partners, order and
    branches); returns the post-collision velocities."""
    n, dim = xs.shape
    r2 = _r2(xs, xs).detach()
    fluid = (types == FLUID).cpu().numpy()
    act = (types != GHOST).cpu().numpy()
    r2n = r2.cpu().numpy()
    if dim == 3:
        cand = mprev.cpu().numpy() & (r2n < c["col2"])
        lin = _cell_lin(key, c)
    else:
        cand = (r2n < c["col2"]) & act[None, :]
        np.fill_diagonal(cand, False)
    events = []
    for i in np.nonzero(fluid)[0]:
        js = np.nonzero(cand[i] & act)[0]
        if len(js) == 0:
            continue
        order = np.lexsort((-js, lin[js])) if dim == 3 else np.argsort(js)
        events.append((i, js[order]))
    v = us.clone()
    if not events:
        return v
    rank = 0
    while True:
        pairs = [(i, js[rank]) for i, js in events if rank < len(js)]
        if not pairs:
            break
        ii = torch.tensor([p[0] for p in pairs], dtype=torch.long, device=xs.device)
        jj = torch.tensor([p[1] for p in pairs], dtype=torch.long, device=xs.device)
        dr = xs[jj] - xs[ii]
        rr = torch.sqrt(torch.sum(dr * dr, dim=1))
        ok = rr >= c["col_rmin"]
        rs = torch.where(ok, rr, torch.ones_like(rr))
        nrm = dr / rs[:, None]
        vn = torch.sum((v[ii] - us[jj]) * nrm, dim=1)
        hit = (ok & (vn > 0.0)).detach()
        upd = v[ii] - (c["half1pe"] * vn)[:, None] * nrm
        v = v.index_put((ii,), torch.where(hit[:, None], upd, v[ii]))
        rank += 1
    return v


def step(x, u, key, types, g, nu, c, drive=None):
    """One step.  x, u: (N, dim) FP64 tensors (may require grad); key: the
    positions of the last neighbour search (previous step's list), no grad;
    types: int tensor; g: (dim,) gravity; nu: scalar viscosity.
    drive: None, or driven walls as dict(amp, freq (tensors), axis, rest
    (N, dim) positions at t = 0, t1 = time at the end of this step): WALL
    and DUMMY particles go to rest + amp sin(2 pi freq t1) along axis with
    the matching velocity after the explicit update, and keep it.
    Returns (x, u, key, types, info) after the step."""
    dim = c["dim"]
    fluid = types == FLUID
    fl = fluid[:, None].to(x.dtype)
    # 1. viscosity on the previous step's list, explicit update
    mprev = _members(key, types, c)
    r2 = _r2(x, x)
    r = _safe_r(r2, mprev)
    w = _kw(r, c["re_lap"], c["rmin"]) * mprev
    lap = torch.stack([torch.sum((u[None, :, d] - u[:, None, d]) * w, dim=1) for d in range(dim)], dim=1)
    a = g[None, :] + (nu * c["coeff"]) * lap
    us = u + c["dt"] * a * fl
    xs = x + c["dt"] * us * fl
    walls = (types == WALL) | (types == DUMMY)
    if drive is not None:
        om = 2.0 * np.pi * drive["freq"]
        ph = om * drive["t1"]
        ax = drive["axis"]
        onehot = torch.zeros(dim, dtype=x.dtype, device=x.device)
        onehot[ax] = 1.0
        xw = drive["rest"] + (drive["amp"] * torch.sin(ph)) * onehot[None, :] + \
            (x - drive["rest"]) * (1.0 - onehot[None, :])
        uw = (drive["amp"] * om * torch.cos(ph)) * onehot[None, :].expand_as(u)
        xs = torch.where(walls[:, None], xw, xs)
        us = torch.where(walls[:, None], uw, us)
    # 2. collision
    if c["col_on"]:
        uc_v = _collision(xs, us, key, types, mprev, c)
        uc = torch.where(fluid[:, None], uc_v, us)
        xc = xs + c["dt"] * (uc - us) * fl
    else:
        uc, xc = us, xs
    # 3. fresh list, density, surface flags
    m = _members(xc.detach(), types, c)
    r2 = _r2(xc, xc)
    r = _safe_r(r2, m)
    n = torch.sum(_kw(r, c["re_n"], c["rmin"]) * m, dim=1)
    with torch.no_grad():
        if c["surf_method"] == 1:
            cnt = torch.sum(((r2 < c["re_n2"]) & m).to(torch.int64), dim=1)
            surf = fluid & (cnt.to(x.dtype) < c["count_thr"])
        else:
            surf = fluid & (n < c["surf_thr"])
    # 4. PPE
    unk = (fluid & ~surf) | (types == WALL)
    nd = types != DUMMY
    wl = _kw(r, c["re_lap"], c["rmin"]) * (m & nd[None, :])
    idx = torch.nonzero(unk).flatten()
    P = torch.zeros_like(n)
    if len(idx):
        wu = wl[idx][:, idx]
        A = -c["coeff"] * wu + torch.diag(c["coeff"] * torch.sum(wl[idx], dim=1))
        b = torch.where(fluid[idx], c["rhs_k"] * (n[idx] - c["n0"]) / c["n0"], torch.zeros_like(n[idx]))
        P = P.index_put((idx,), torch.linalg.solve(A, b))
    # 5. P_min and gradient
    Pj = torch.where(m, P[None, :].expand_as(r), torch.full_like(r, float("inf")))
    pmin = torch.minimum(P, torch.min(Pj, dim=1).values)
    mg = m & (r2 >= c["grad_r2min"])
    rg = _safe_r(r2, mg)
    wg = _kw(rg, c["re_lap"], c["rmin"]) * mg
    coef = (P[None, :] - pmin[:, None]) / torch.where(mg, r2, torch.ones_like(r2)) * wg
    gsum = torch.stack([torch.sum(coef * (xc[None, :, d] - xc[:, None, d]), dim=1) for d in range(dim)], dim=1)
    acc = c["neg_grad"] * gsum / c["density"]
    du = c["dt"] * acc * fl
    un = uc + du
    xn = xc + c["dt"] * du
    # 6. walls, out of bounds
    with torch.no_grad():
        lo = torch.tensor(c["oob_lo"], dtype=x.dtype, device=x.device)
        hi = torch.tensor(c["oob_hi"], dtype=x.dtype, device=x.device)
        out = fluid & (torch.any((xn < lo) | (xn > hi), dim=1) | torch.any(torch.isnan(xn), dim=1))
        ntypes = torch.where(out, torch.full_like(types, GHOST), types)
    still = (ntypes == FLUID)[:, None]
    if drive is not None:
        still = still | walls[:, None]
    un = torch.where(still, un, torch.zeros_like(un))
    info = dict(P=P, n=n, surf=surf, unknown=unk)
    return xn, un, xc.detach(), ntypes, info
