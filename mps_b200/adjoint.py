"""Differentiation form: a multi-step MPS rollout as a differentiable
function for ``torch.autograd``, over the session C ABI.

``Rollout(cfg, dim, pos, types, steps, every)`` binds one session to a fixed
initial geometry; calling it with an initial velocity field ``u0`` (n, dim),
a gravity scale, a kinematic viscosity and, for driven walls, the drive's
amplitude and frequency (torch FP64 tensors) runs ``steps`` device-resident
time steps and returns the final positions and velocities (n, dim) in
reference order.  With ``probe`` (particle indices or a boolean mask in
reference order, e.g. the wall particles of a pressure probe) it also
returns the probe's mean pressure after every step, a (steps,) series that
a loss may use (the sloshing case's time-mean squared wall pressure); its
adjoint enters each reversed step through mps_adjoint_pressure_seed.
Backward runs the hand-written
adjoint kernels of the library (``mps_step_adjoint``) from the last step to
the first with checkpoint-every-k recomputation: the forward saves the
state every ``every`` steps; the backward reloads each checkpoint, recomputes
its segment saving the state at every step, and reverses the segment's
steps from those states.  Memory: steps/every + every states.

Discrete decisions of each step (neighbour sets, collision branches,
free-surface flags, the PPE unknown set, P_min's argument, ghosting) are
held fixed, so the gradient is that of the piecewise-smooth map on the
forward run's branch.  n0 and lambda are computed once from the initial
positions and held constant.  The reference has no adjoint; the checks are
central finite differences and a dense FP64 autograd of the same step.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .session import Session
from .types import HostParticles


class Rollout:
    def __init__(self, cfg, dim: int, pos, types, steps: int, every: int = 1, precision: int = _lib.PREC_FP64,
                 checkpoint_device: str | None = None, drive_axis: int = 0, probe=None):
        if steps < 1 or every < 1:
            raise ValueError("steps and every must be positive")
        self.cfg, self.dim, self.steps, self.every = cfg, dim, int(steps), int(every)
        self.pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, dim)
        self.types = np.ascontiguousarray(types, dtype=np.int32)
        self.n = self.types.shape[0]
        self.probe = None
        if probe is not None:
            pr = np.asarray(probe)
            if pr.dtype == bool:
                if pr.shape != (self.n,):
                    raise ValueError("a boolean probe needs one entry per particle")
                self.probe = np.flatnonzero(pr)
            else:
                self.probe = pr.astype(np.int64).ravel()
            if self.probe.size == 0:
                raise ValueError("the probe selects no particle")
            if self.probe.min() < 0 or self.probe.max() >= self.n:
                raise ValueError("probe index out of range")
        self.series = np.zeros(0)
        self.sess = Session(cfg, dim, self.n, precision=precision)
        self.g_base = np.array([cfg.gravity[d] for d in range(dim)], dtype=np.float64)
        self.drive_axis = int(drive_axis)
        self._upload(np.zeros_like(self.pos))
        self.n0, self.lam, self.n0_count = self.sess.compute_initial_params()
        self.nbytes = self.sess.state_bytes()
        if checkpoint_device is None:
            checkpoint_device = "cuda" if torch.cuda.is_available() else "cpu"
        self.ck_device = checkpoint_device

    # ---- plumbing ----------------------------------------------------------------
    def _upload(self, u0: np.ndarray):
        hp = HostParticles(self.dim, self.pos, u0, self.types)
        self.sess.upload(hp)

    def _set_params(self, gscale: float, nu: float, amp: float = 0.0, freq: float = 0.0):
        p = self.sess.params
        for d in range(self.dim):
            p.gravity[d] = float(self.g_base[d] * gscale)
        p.viscosity = float(nu)
        p.wall_drive_amp = float(amp)
        p.wall_drive_freq = float(freq)
        p.wall_drive_axis = self.drive_axis
        self.sess._check(self.sess.lib.mps_update_params(self.sess.h, p))

    def _buffer(self) -> torch.Tensor:
        return torch.empty(self.nbytes, dtype=torch.uint8, device=self.ck_device)

    def _save(self) -> torch.Tensor:
        b = self._buffer()
        self.sess.state_save(b.data_ptr())
        return b

    def _final(self):
        out = self.sess.download()
        return out["pos"].copy(), out["vel"].copy(), out["type"].copy()

    # ---- forward / backward ---------------------------------------------------------
    def forward(self, u0: np.ndarray, gscale: float, nu: float, amp: float = 0.0, freq: float = 0.0):
        """Run the rollout; returns (x_T, u_T, types_T) and keeps the checkpoints."""
        self._set_params(gscale, nu, amp, freq)
        self._upload(u0)
        self.sess.set_initial_params(self.n0, self.lam, self.n0_count)
        self.sess.neighbor_search()
        self.ckpts = []
        self.series = np.zeros(self.steps if self.probe is not None else 0)
        for s in range(self.steps):
            if s % self.every == 0:
                self.ckpts.append(self._save())
            self.sess.step(1)
            if self.probe is not None:
                self.series[s] = self.sess.pressure()[self.probe].mean()
        return self._final()

    def backward(self, lam_x: np.ndarray, lam_u: np.ndarray, lam_series: np.ndarray | None = None):
        """Adjoint of the last forward run from the adjoint of (x_T, u_T)
        and, with a probe, of the probe pressure series: returns (dL/dx_0,
        dL/du_0, dL/d gravity_scale, dL/d viscosity, dL/d drive amplitude,
        dL/d drive frequency)."""
        if lam_series is not None and self.probe is None:
            raise ValueError("lam_series needs a Rollout with a probe")
        self.sess.adjoint_seed(lam_x, lam_u)
        nseg = len(self.ckpts)
        for seg in reversed(range(nseg)):
            s0 = seg * self.every
            s1 = min(s0 + self.every, self.steps)
            self.sess.state_load(self.ckpts[seg].data_ptr())
            states = [self.ckpts[seg]]
            for _ in range(s0, s1 - 1):
                self.sess.step(1)
                states.append(self._save())
            for k in reversed(range(s1 - s0)):
                self.sess.state_load(states[k].data_ptr())
                if lam_series is not None and lam_series[s0 + k] != 0.0:
                    seed = np.zeros(self.n)
                    seed[self.probe] = lam_series[s0 + k] / self.probe.size
                    self.sess.adjoint_pressure_seed(seed)
                self.sess.step_adjoint()
        lx, lu, gg, gn, gd = self.sess.adjoint_get()
        return lx, lu, float(np.dot(gg, self.g_base)), gn, float(gd[0]), float(gd[1])

    def close(self):
        self.sess.close()

    def __call__(self, u0: torch.Tensor, gscale: torch.Tensor, nu: torch.Tensor, amp: torch.Tensor | None = None,
                 freq: torch.Tensor | None = None):
        z = torch.zeros((), dtype=torch.float64, device=u0.device)
        out = _RolloutFn.apply(u0, gscale, nu, z if amp is None else amp, z if freq is None else freq, self)
        return out if self.probe is not None else out[:2]


class _RolloutFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, gscale, nu, amp, freq, roll):
        x, u, t = roll.forward(u0.detach().cpu().numpy(), float(gscale), float(nu), float(amp), float(freq))
        ctx.roll = roll
        ctx.dev = u0.device
        return (torch.from_numpy(x).to(ctx.dev), torch.from_numpy(u).to(ctx.dev),
                torch.from_numpy(roll.series.copy()).to(ctx.dev))

    @staticmethod
    def backward(ctx, gx, gu, gs):
        roll = ctx.roll
        lx = np.zeros((roll.n, roll.dim)) if gx is None else gx.detach().cpu().numpy()
        lu = np.zeros((roll.n, roll.dim)) if gu is None else gu.detach().cpu().numpy()
        ls = None if (gs is None or roll.probe is None) else gs.detach().cpu().numpy()
        _, du0, dgs, dnu, da, df = roll.backward(lx, lu, ls)
        f64 = dict(dtype=torch.float64, device=ctx.dev)
        return (torch.from_numpy(du0).to(ctx.dev), torch.tensor(dgs, **f64), torch.tensor(dnu, **f64),
                torch.tensor(da, **f64), torch.tensor(df, **f64), None)
