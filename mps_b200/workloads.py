"""Seeded dam-break workloads in the reference solver's input conventions.

The lattice rules follow the reference's initial-condition generators
(3-D: ``mps_fluid3D/tools/gen_dambreak.py:105-166``; 2-D:
``mps_fluid2D/tools/gen_dambreak.py:108-156``): particles on a square lattice
of spacing l0, wall on or beyond the tank faces (bottom, sides, front/back;
no lid), dummy beyond ``wall_layers`` layers, fluid inside the water column.
On top of that this module adds a seeded uniform jitter of +-jitter*l0 per
axis on FLUID particles only (numpy ``PCG64(seed)``), optional seeded
Gaussian initial velocities, and writes positions with ``%.17e`` so every
reader sees the same bits.

Named workloads (sizes are produced by these rules):

=======  ====  ==============================================  ======  =====
name     dim   geometry                                          l0      dt
=======  ====  ==============================================  ======  =====
c0       2     tank 1.0 x 0.6, column 0.25 x 0.5                 0.01    1e-3
c1       3     tank 1.6 x 0.6 x 0.6, column 0.4 x 0.6 x 0.3      0.005   5e-4
c2       3     as c1                                            0.0035  3.5e-4
c3       2     as c0                                            0.005   5e-4
=======  ====  ==============================================  ======  =====
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

from .types import DUMMY, FLUID, WALL

EPS = 1.0e-10


def dambreak3d_lattice(l0, domain, water, wall_layers=2, dummy_layers=2):
    """Unjittered 3-D lattice in the reference generator's loop order (i, j, k)."""
    dx, dy, dz = domain
    wx, wy, wz = water
    wl, dl = wall_layers, dummy_layers
    tl = wl + dl
    i_right = int(dx / l0)
    k_back = int(dz / l0)
    i_r = np.arange(-(tl - 1), i_right + (tl - 1) + 1)
    j_r = np.arange(-(tl - 1), int(dy / l0) + 1)
    k_r = np.arange(-(tl - 1), k_back + (tl - 1) + 1)
    I, J, K = np.meshgrid(i_r, j_r, k_r, indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    x, y, z = I * l0, J * l0, K * l0
    t = np.full(I.shape, -1, dtype=np.int32)
    wall = (J <= 0) | (I <= 0) | (I >= i_right) | (K <= 0) | (K >= k_back)
    t[wall] = WALL
    dummy = (J <= -wl) | (I <= -wl) | (I >= i_right + wl) | (K <= -wl) | (K >= k_back + wl)
    t[dummy] = DUMMY
    fluid = (t < 0) & (I >= 1) & (x <= wx + EPS) & (J >= 1) & (y <= wy + EPS) & (K >= 1) & (z <= wz + EPS)
    t[fluid] = FLUID
    keep = t >= 0
    pos = np.stack([x[keep], y[keep], z[keep]], axis=1).astype(np.float64)
    return pos, t[keep]


def dambreak2d_lattice(l0, domain, water, wall_layers=2, dummy_layers=2):
    """Unjittered 2-D lattice in the reference generator's loop order (i, j)."""
    dx, dy = domain
    wx, wy = water
    wl, dl = wall_layers, dummy_layers
    tl = wl + dl
    i_right = int(round(dx / l0))
    i_r = np.arange(-(tl - 1), i_right + (tl - 1) + 1)
    j_r = np.arange(-(tl - 1), int(round(dy / l0)) + 1)
    I, J = np.meshgrid(i_r, j_r, indexing="ij")
    I, J = I.ravel(), J.ravel()
    x, y = I * l0, J * l0
    t = np.full(I.shape, -1, dtype=np.int32)
    t[(J <= 0) | (I <= 0) | (I >= i_right)] = WALL
    t[(J <= -wl) | (I <= -wl) | (I >= i_right + wl)] = DUMMY
    fluid = (t < 0) & (I >= 1) & (x <= wx + EPS) & (J >= 1) & (y <= wy + EPS)
    t[fluid] = FLUID
    keep = t >= 0
    pos = np.stack([x[keep], y[keep]], axis=1).astype(np.float64)
    return pos, t[keep]


def jitter_fluid(pos, types, l0, frac, seed):
    """Uniform +-frac*l0 per axis on fluid particles, drawn in particle order."""
    pos = pos.copy()
    if frac > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        f = types == FLUID
        pos[f] += rng.uniform(-frac * l0, frac * l0, size=(int(f.sum()), pos.shape[1]))
    return pos


def common_params(dim: int, l0: float, dt: float, steps: int, domain) -> dict:
    """Parameter set shared by the named workloads (reference key names)."""
    p = {
        "particle_distance": repr(l0),
        "influence_ratio_lap": "3.1",
        "influence_ratio_n": "2.1",
        "max_neighbors": "512",
        "wall_layers": "2",
        "dummy_layers": "2",
        "density": "1000.0",
        "viscosity": "1e-06",
        "gravity_x": "0.0",
        "gravity_y": "-9.81",
        "dt": repr(dt),
        "t_end": repr((steps + 0.5) * dt),
        "output_interval": str(10**9),
        "solver_type": "1",
        "cg_max_iter": "10000",
        "cg_tolerance": "1e-9",
        "relaxation_coeff": "0.2",
        "clamp_negative_pressure": "0",
        "ppe_type": "0",
        "hs_mode": "0",
        "cmps_gradient": "0",
        "use_analytical_lambda": "0",
        "surface_threshold": "0.97",
        "surface_detection_method": "0",
        "restitution_coeff": "0.2",
        "collision_distance_ratio": "0.5",
        "domain_x_min": "0.0",
        "domain_x_max": repr(domain[0]),
        "domain_y_min": "0.0",
        "domain_y_max": repr(domain[1]),
    }
    if dim == 3:
        p["gravity_z"] = "0.0"
        p["domain_z_min"] = "0.0"
        p["domain_z_max"] = repr(domain[2])
    return p


@dataclass
class Workload:
    name: str
    dim: int
    pos: np.ndarray
    vel: np.ndarray
    types: np.ndarray
    params: dict = field(default_factory=dict)
    steps: int = 1
    # driven walls (amplitude m, frequency Hz, axis); not a reference deck key,
    # set on the session parameters (mps_params_t.wall_drive_*)
    drive: tuple = (0.0, 0.0, 0)

    @property
    def n(self):
        return int(self.pos.shape[0])

    @property
    def n_fluid(self):
        return int((self.types == FLUID).sum())

    def config(self):
        """SimConfig built exactly as the reference's parser would from params.txt."""
        from .config import config_apply, config_derive_radii, config_set_defaults

        cfg = config_set_defaults(self.dim)
        for k, v in self.params.items():
            config_apply(cfg, k, v, self.dim)
        config_derive_radii(cfg)
        return cfg

    def write(self, outdir: str, fmt: str = "%.17e") -> str:
        """Write particles.txt / params.txt / cal.txt; returns the cal.txt path."""
        os.makedirs(outdir, exist_ok=True)
        write_particles(os.path.join(outdir, "particles.txt"), self.pos, self.vel, self.types, fmt,
                        header=f"# {self.name}: {self.n} particles, {self.n_fluid} fluid")
        with open(os.path.join(outdir, "params.txt"), "w") as fh:
            fh.write(f"# {self.name}\n")
            for k, v in self.params.items():
                fh.write(f"{k} {v}\n")
            fh.write("output_dir output\n")
        cal = os.path.join(outdir, "cal.txt")
        with open(cal, "w") as fh:
            fh.write("particle_file particles.txt\nparam_file params.txt\n")
        return cal


def write_particles(path, pos, vel, types, fmt="%.17e", header=""):
    n, dim = pos.shape
    with open(path, "w") as fh:
        if header:
            fh.write(header.rstrip("\n") + "\n")
        fh.write(f"{n}\n")
        fh.write("# x y " + ("z " if dim == 3 else "") + "vx vy " + ("vz " if dim == 3 else "") + "type\n")
        cols = np.concatenate([pos, vel], axis=1)
        line_fmt = " ".join([fmt] * (2 * dim)) + " %d"
        np.savetxt(fh, np.column_stack([cols, types]), fmt=line_fmt.split(" "), delimiter=" ")


def dambreak(name: str, seed: int = 0, jitter: float = 0.01, vel_sigma: float = 0.0,
             l0: float | None = None, steps: int | None = None, gravity_scale: float = 1.0) -> Workload:
    """Build a named workload (c0..c3) or a scaled variant (l0 override)."""
    specs = {
        "c0": (2, 0.01, 1.0e-3, 1000, (1.0, 0.6), (0.25, 0.5)),
        "c1": (3, 0.005, 5.0e-4, 1000, (1.6, 0.6, 0.6), (0.4, 0.6, 0.3)),
        "c2": (3, 0.0035, 3.5e-4, 1000, (1.6, 0.6, 0.6), (0.4, 0.6, 0.3)),
        "c3": (2, 0.005, 5.0e-4, 200, (1.0, 0.6), (0.25, 0.5)),
    }
    dim, l0d, dt, nsteps, domain, water = specs[name]
    l0 = l0d if l0 is None else l0
    nsteps = nsteps if steps is None else steps
    if dim == 3:
        pos, t = dambreak3d_lattice(l0, domain, water)
    else:
        pos, t = dambreak2d_lattice(l0, domain, water)
    pos = jitter_fluid(pos, t, l0, jitter, seed)
    vel = np.zeros_like(pos)
    if vel_sigma > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed + 1))
        f = t == FLUID
        vel[f] = rng.normal(0.0, vel_sigma, size=(int(f.sum()), dim))
    params = common_params(dim, l0, dt, nsteps, domain)
    if gravity_scale != 1.0:
        params["gravity_y"] = repr(-9.81 * gravity_scale)
    suffix = "" if l0 == l0d else f"@l0={l0}"
    return Workload(name + suffix, dim, pos, vel, t, params, nsteps)


def sloshing3d(l0: float = 0.004, seed: int = 0, jitter: float = 0.01, amp: float = 0.01, freq: float = 1.5,
               steps: int = 500, dt: float = 4.0e-4, domain=(0.6, 0.4, 0.3), depth: float = 0.2) -> Workload:
    """3-D sloshing: tank 0.6 x 0.4 x 0.3 m (y vertical) filled to `depth`,
    walls driven sinusoidally along x (amplitude `amp`, frequency `freq`),
    the dam break's lattice rules and parameters otherwise."""
    water = (domain[0], depth, domain[2])
    pos, t = dambreak3d_lattice(l0, domain, water)
    pos = jitter_fluid(pos, t, l0, jitter, seed)
    params = common_params(3, l0, dt, steps, domain)
    return Workload(f"sloshing3d@l0={l0}", 3, pos, np.zeros_like(pos), t, params, steps, drive=(amp, freq, 0))


def small_dambreak3d(l0: float = 0.02, seed: int = 0, jitter: float = 0.01,
                     domain=(0.4, 0.3, 0.2), water=(0.1, 0.2, 0.2), dt: float = 5.0e-4,
                     steps: int = 10, **overrides) -> Workload:
    """A few thousand particles: quick parity cases with the named workloads' parameters."""
    pos, t = dambreak3d_lattice(l0, domain, water)
    pos = jitter_fluid(pos, t, l0, jitter, seed)
    params = common_params(3, l0, dt, steps, domain)
    params.update({k: str(v) for k, v in overrides.items()})
    return Workload(f"small3d@l0={l0}", 3, pos, np.zeros_like(pos), t, params, steps)


def small_dambreak2d(l0: float = 0.02, seed: int = 0, jitter: float = 0.01,
                     domain=(1.0, 0.6), water=(0.25, 0.5), dt: float = 1.0e-3,
                     steps: int = 10, **overrides) -> Workload:
    pos, t = dambreak2d_lattice(l0, domain, water)
    pos = jitter_fluid(pos, t, l0, jitter, seed)
    params = common_params(2, l0, dt, steps, domain)
    params.update({k: str(v) for k, v in overrides.items()})
    return Workload(f"small2d@l0={l0}", 2, pos, np.zeros_like(pos), t, params, steps)


def example_dambreak3d() -> Workload:
    """The reference's shipped 3-D example deck (examples/dambreak): l0 0.008,
    tank 0.584 x 0.292 x 0.024, column 0.146 x 0.292 x 0.024, no jitter, with
    its parameter file's values (hs_mode 1, negative-pressure clamp, re 2.1 l0,
    tolerance 1e-8)."""
    L = 0.146
    domain = (L * 4, L * 2, 0.024)
    water = (L, L * 2, 0.024)
    pos, t = dambreak3d_lattice(0.008, domain, water)
    # The shipped deck stores positions with %.8e; the reference reads those.
    pos = np.array([float("%.8e" % x) for x in pos.ravel()]).reshape(pos.shape)
    params = common_params(3, 0.008, 5.0e-4, 4000, domain)
    params.update({
        "influence_ratio_lap": "2.1",
        "hs_mode": "1",
        "clamp_negative_pressure": "1",
        "cg_tolerance": "1.0e-8",
        "t_end": "2.0",
        "output_interval": "100",
    })
    return Workload("example_dambreak3d", 3, pos, np.zeros_like(pos), t, params, 4000)
