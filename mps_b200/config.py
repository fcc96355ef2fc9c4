"""Parameter files of the reference solver, parsed with the reference's rules.

* ``config_set_defaults``  <- mps_fluid3D_parallel/src/sim_config.c:20-79
  (2-D: mps_fluid2D/src/sim_config.c, which differs in ``max_neighbors`` 256,
  the domain default and the absent z fields)
* ``config_load_cal``      <- sim_config.c:86-159 (paths relative to cal.txt)
* ``config_load_params``   <- sim_config.c:166-277 (``key value`` lines, ``#``
  comments, unknown keys warn, radii derived after parsing)

Values are converted like C's ``atof``/``atoi``: the longest numeric prefix
counts and garbage yields 0.
"""
from __future__ import annotations

import os
import re
import sys

from .types import sim_config_type

_FLOAT_PREFIX = re.compile(
    r"\s*[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)", re.IGNORECASE
)
_INT_PREFIX = re.compile(r"\s*[+-]?\d+")


def c_atof(s: str) -> float:
    m = _FLOAT_PREFIX.match(s)
    return float(m.group(0)) if m else 0.0


def c_atoi(s: str) -> int:
    m = _INT_PREFIX.match(s)
    if not m:
        return 0
    v = int(m.group(0))
    return ((v + 2**31) % 2**32) - 2**31


def config_set_defaults(dim: int = 3):
    cfg = sim_config_type(dim)()
    cfg.particle_distance = 0.025
    cfg.influence_ratio_lap = 2.1
    cfg.influence_radius_lap = 2.1 * 0.025
    cfg.influence_ratio_n = 2.1
    cfg.influence_radius_n = 2.1 * 0.025
    cfg.max_neighbors = 512 if dim == 3 else 256
    cfg.wall_layers = 2
    cfg.dummy_layers = 2
    cfg.density = 1000.0
    cfg.viscosity = 1.0e-6
    cfg.gravity[0] = 0.0
    cfg.gravity[1] = -9.81
    if dim == 3:
        cfg.gravity[2] = 0.0
    cfg.dt = 5.0e-4
    cfg.t_end = 2.0
    cfg.output_interval = 100
    cfg.solver_type = 0
    cfg.cg_max_iter = 10000
    cfg.cg_tolerance = 1.0e-8
    cfg.relaxation_coeff = 0.2
    cfg.clamp_negative_pressure = 0
    cfg.ppe_type = 0
    cfg.c_ppe = 1.01
    cfg.gamma_ppe = 0.01
    cfg.surface_threshold = 0.97
    cfg.surface_detection_method = 0
    cfg.surface_count_threshold = 0.85
    cfg.restitution_coeff = 0.2
    cfg.collision_distance_ratio = 0.5
    cfg.surface_tension_enabled = 0
    cfg.surface_tension_coeff = 0.0728
    cfg.surface_tension_re_ratio = 3.2
    cfg.influence_radius_st = 3.2 * 0.025
    cfg.wetting_angle_SL = 90.0
    for d in range(dim):
        cfg.domain_min[d] = 0.0
    if dim == 3:
        cfg.domain_max[0], cfg.domain_max[1], cfg.domain_max[2] = 0.4, 0.3, 0.2
    else:
        cfg.domain_max[0], cfg.domain_max[1] = 1.0, 0.6
    cfg.cmps_gradient = 0
    cfg.use_analytical_lambda = 0
    cfg.hs_mode = 0
    cfg.output_dir = b"output"
    return cfg


def _resolve(cal_path: str, value: str) -> str:
    if value.startswith("/"):
        return value[:255]
    d = cal_path[:255]
    k = d.rfind("/")
    return (d[: k + 1] + value)[:255] if k >= 0 else value[:255]


def _two_tokens(line: str):
    s = line.strip()
    if not s or s.startswith("#"):
        return None
    parts = s.split()
    if len(parts) < 2:
        return None
    return parts[0][:127], parts[1][:255]


def config_load_cal(cal_path: str, cfg) -> int:
    try:
        fh = open(cal_path, "r", errors="replace")
    except OSError:
        print(f"Error: cannot open cal file '{cal_path}'", file=sys.stderr)
        return -1
    with fh:
        for line in fh:
            kv = _two_tokens(line)
            if kv is None:
                continue
            key, value = kv
            if key == "particle_file":
                cfg.particle_file = _resolve(cal_path, value).encode()
            elif key == "param_file":
                cfg.param_file = _resolve(cal_path, value).encode()
            else:
                print(f"Warning: unknown key in cal file: '{key}'", file=sys.stderr)
    if not cfg.particle_file:
        print(f"Error: particle_file not specified in '{cal_path}'", file=sys.stderr)
        return -1
    if not cfg.param_file:
        print(f"Error: param_file not specified in '{cal_path}'", file=sys.stderr)
        return -1
    return 0


def _param_table(dim: int):
    f, i = c_atof, c_atoi
    t = {
        "particle_distance": ("particle_distance", f),
        "influence_ratio_lap": ("influence_ratio_lap", f),
        "influence_ratio_n": ("influence_ratio_n", f),
        "max_neighbors": ("max_neighbors", i),
        "wall_layers": ("wall_layers", i),
        "dummy_layers": ("dummy_layers", i),
        "density": ("density", f),
        "viscosity": ("viscosity", f),
        "gravity_x": (("gravity", 0), f),
        "gravity_y": (("gravity", 1), f),
        "dt": ("dt", f),
        "t_end": ("t_end", f),
        "output_interval": ("output_interval", i),
        "solver_type": ("solver_type", i),
        "cg_max_iter": ("cg_max_iter", i),
        "cg_tolerance": ("cg_tolerance", f),
        "relaxation_coeff": ("relaxation_coeff", f),
        "clamp_negative_pressure": ("clamp_negative_pressure", i),
        "ppe_type": ("ppe_type", i),
        "c_ppe": ("c_ppe", f),
        "gamma_ppe": ("gamma_ppe", f),
        "surface_threshold": ("surface_threshold", f),
        "surface_detection_method": ("surface_detection_method", i),
        "surface_count_threshold": ("surface_count_threshold", f),
        "restitution_coeff": ("restitution_coeff", f),
        "collision_distance_ratio": ("collision_distance_ratio", f),
        "surface_tension_enabled": ("surface_tension_enabled", i),
        "surface_tension_coeff": ("surface_tension_coeff", f),
        "surface_tension_re_ratio": ("surface_tension_re_ratio", f),
        "wetting_angle_SL": ("wetting_angle_SL", f),
        "domain_x_min": (("domain_min", 0), f),
        "domain_x_max": (("domain_max", 0), f),
        "domain_y_min": (("domain_min", 1), f),
        "domain_y_max": (("domain_max", 1), f),
        "cmps_gradient": ("cmps_gradient", i),
        "use_analytical_lambda": ("use_analytical_lambda", i),
        "hs_mode": ("hs_mode", i),
    }
    if dim == 3:
        # the 3-D serial variant's friction keys (mps_fluid3D/src/sim_config.c:267-274),
        # kept as attributes of the config: the OpenMP layout has no such fields
        t["friction_enabled"] = ("friction_enabled", i)
        t["friction_delta_theta"] = ("friction_delta_theta", f)
        t["dynamic_friction_alpha"] = ("dynamic_friction_alpha", f)
        t["friction_velocity_threshold"] = ("friction_velocity_threshold", f)
        t["gravity_z"] = (("gravity", 2), f)
        t["domain_z_min"] = (("domain_min", 2), f)
        t["domain_z_max"] = (("domain_max", 2), f)
    return t


def config_derive_radii(cfg) -> None:
    """sim_config.c:271-274: radii follow the ratios after parsing."""
    cfg.influence_radius_lap = cfg.influence_ratio_lap * cfg.particle_distance
    cfg.influence_radius_n = cfg.influence_ratio_n * cfg.particle_distance
    cfg.influence_radius_st = cfg.surface_tension_re_ratio * cfg.particle_distance


def config_apply(cfg, key: str, value: str, dim: int) -> bool:
    """Apply one ``key value`` pair; False (and a warning) for unknown keys."""
    if key == "output_dir":
        cfg.output_dir = value.encode()[:255]
        return True
    ent = _param_table(dim).get(key)
    if ent is None:
        print(f"Warning: unknown parameter '{key}'", file=sys.stderr)
        return False
    field, conv = ent
    if isinstance(field, tuple):
        getattr(cfg, field[0])[field[1]] = conv(value)
    else:
        setattr(cfg, field, conv(value))
    return True


def config_load_params(param_path: str, cfg, dim: int = 3) -> int:
    try:
        fh = open(param_path, "r", errors="replace")
    except OSError:
        print(f"Error: cannot open param file '{param_path}'", file=sys.stderr)
        return -1
    with fh:
        for line in fh:
            kv = _two_tokens(line)
            if kv is not None:
                config_apply(cfg, kv[0], kv[1], dim)
    config_derive_radii(cfg)
    return 0


def load_deck(cal_path: str, dim: int = 3):
    """Defaults, then cal.txt, then params.txt -- main.c:98-104 of the reference."""
    cfg = config_set_defaults(dim)
    if config_load_cal(cal_path, cfg) != 0:
        raise ValueError(f"cannot load cal file {cal_path}")
    if config_load_params(cfg.param_file.decode(), cfg, dim) != 0:
        raise ValueError(f"cannot load params file {cfg.param_file.decode()}")
    return cfg


def neighbor_radius(cfg) -> float:
    """simulation.c:22-24: the list radius is the largest active radius."""
    re = max(cfg.influence_radius_lap, cfg.influence_radius_n)
    if cfg.surface_tension_enabled:
        re = max(re, cfg.influence_radius_st)
    return re


def load_particles(path: str, dim: int = 3):
    """main.c:20-85: header count after comments, then ``x y [z] vx vy [vz] type`` lines.

    Returns (pos, vel, type) numpy arrays.  Malformed lines are skipped with a
    warning, as in the reference; there is no capacity limit here.
    """
    import numpy as np

    with open(path, "r", errors="replace") as fh:
        lines = fh.read().splitlines()
    it = iter(lines)
    count = None
    for line in it:
        s = line.lstrip(" \t")
        if not s or s[0] in "#\r":
            continue
        m = _INT_PREFIX.match(s)
        if m:
            count = int(m.group(0))
            break
    if count is None or count <= 0:
        raise ValueError(f"invalid particle count in '{path}'")
    ncol = 2 * dim + 1
    rows = []
    for line in it:
        if len(rows) >= count:
            break
        s = line.lstrip(" \t")
        if not s or s[0] in "#\r":
            continue
        tok = s.split()
        try:
            vals = [float(t) for t in tok[: ncol - 1]] + [int(tok[ncol - 1])]
            if len(tok) < ncol:
                raise ValueError
        except (ValueError, IndexError):
            print(f"Warning: skipping malformed line: {line}", file=sys.stderr)
            continue
        rows.append(vals)
    if len(rows) != count:
        print(f"Warning: expected {count} particles but loaded {len(rows)}", file=sys.stderr)
    a = np.array([r[: ncol - 1] for r in rows], dtype=np.float64).reshape(-1, ncol - 1)
    t = np.array([r[ncol - 1] for r in rows], dtype=np.int32)
    return a[:, :dim].copy(), a[:, dim:].copy(), t


def abspath_in(dirname: str, name: str) -> str:
    return os.path.join(dirname, name)
