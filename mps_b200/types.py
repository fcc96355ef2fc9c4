"""ctypes / numpy mirrors of the particle data model in ``include/mps_types.h``.

The layouts are the reference solver's ABI (``mps_fluid3D_parallel/include/
particle.h:7-30``, ``neighbor_search.h:8-30``, ``sim_config.h:10-78``; the 2-D
variant differs only through ``DIM``), so the same buffers can be handed to
the CUDA library, to the CPU oracle and to the reference compiled from source.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

FLUID, WALL, GHOST, DUMMY = 0, 1, 2, 3


def particle_dtype(dim: int) -> np.dtype:
    """numpy view of ``Particle`` (104 bytes in 3-D, 80 bytes in 2-D)."""
    return np.dtype(
        [
            ("pos", "f8", (dim,)),
            ("vel", "f8", (dim,)),
            ("acc", "f8", (dim,)),
            ("pressure", "f8"),
            ("n", "f8"),
            ("neighbor_count", "i4"),
            ("type", "i4"),
            ("on_surface", "i4"),
        ],
        align=True,
    )


class ParticleSystem(C.Structure):
    _fields_ = [
        ("particles", C.c_void_p),
        ("num", C.c_int),
        ("capacity", C.c_int),
        ("n0", C.c_double),
        ("lambda_", C.c_double),
        ("C_LL", C.c_double),
        ("C_SL", C.c_double),
        ("n0_count", C.c_int),
    ]


class NeighborList(C.Structure):
    _fields_ = [
        ("neighbors", C.POINTER(C.c_int)),
        ("count", C.POINTER(C.c_int)),
        ("max_neighbors", C.c_int),
    ]


def _cell_list_type(dim: int):
    fields = [
        ("head", C.POINTER(C.c_int)),
        ("next", C.POINTER(C.c_int)),
        ("nx", C.c_int),
        ("ny", C.c_int),
    ]
    if dim == 3:
        fields.append(("nz", C.c_int))
    fields += [
        ("total_cells", C.c_int),
        ("cell_size", C.c_double),
        ("origin", C.c_double * dim),
    ]
    return type(f"CellList{dim}", (C.Structure,), {"_fields_": fields})


def _sim_config_type(dim: int):
    d = C.c_double
    i = C.c_int
    fields = [
        ("particle_distance", d),
        ("influence_ratio_lap", d),
        ("influence_radius_lap", d),
        ("influence_ratio_n", d),
        ("influence_radius_n", d),
        ("max_neighbors", i),
        ("wall_layers", i),
        ("dummy_layers", i),
        ("density", d),
        ("viscosity", d),
        ("gravity", d * dim),
        ("dt", d),
        ("t_end", d),
        ("output_interval", i),
        ("solver_type", i),
        ("cg_max_iter", i),
        ("cg_tolerance", d),
        ("relaxation_coeff", d),
        ("clamp_negative_pressure", i),
        ("ppe_type", i),
        ("c_ppe", d),
        ("gamma_ppe", d),
        ("surface_threshold", d),
        ("surface_detection_method", i),
        ("surface_count_threshold", d),
        ("restitution_coeff", d),
        ("collision_distance_ratio", d),
        ("surface_tension_enabled", i),
        ("surface_tension_coeff", d),
        ("surface_tension_re_ratio", d),
        ("influence_radius_st", d),
        ("wetting_angle_SL", d),
        ("domain_min", d * dim),
        ("domain_max", d * dim),
        ("cmps_gradient", i),
        ("use_analytical_lambda", i),
        ("hs_mode", i),
        ("output_dir", C.c_char * 256),
        ("particle_file", C.c_char * 256),
        ("param_file", C.c_char * 256),
    ]
    return type(f"SimConfig{dim}", (C.Structure,), {"_fields_": fields})


def _serial_config_type():
    """SimConfig of the 3-D serial variant (mps_fluid3D/include/sim_config.h):
    the OpenMP layout with four friction fields after hs_mode."""
    fields = []
    for name, t in _sim_config_type(3)._fields_:
        fields.append((name, t))
        if name == "hs_mode":
            fields += [("friction_enabled", C.c_int), ("friction_delta_theta", C.c_double),
                       ("dynamic_friction_alpha", C.c_double), ("friction_velocity_threshold", C.c_double)]
    return type("SimConfig3S", (C.Structure,), {"_fields_": fields})


FRICTION_DEFAULTS = {"friction_enabled": 0, "friction_delta_theta": 30.0, "dynamic_friction_alpha": 600.0,
                     "friction_velocity_threshold": 0.01}   # mps_fluid3D/src/sim_config.c:76-79


def serial_config(cfg):
    """A SimConfig3S copy of a 3-D config; the friction fields come from the
    config's attributes of the same names, else the serial variant's defaults."""
    out = SimConfig3S()
    for name, _ in SimConfig3._fields_:
        setattr(out, name, getattr(cfg, name))
    for name, v in FRICTION_DEFAULTS.items():
        setattr(out, name, getattr(cfg, name, v))
    return out


CellList3 = _cell_list_type(3)
CellList2 = _cell_list_type(2)
SimConfig3 = _sim_config_type(3)
SimConfig2 = _sim_config_type(2)
SimConfig3S = _serial_config_type()


def sim_config_type(dim: int):
    return SimConfig3 if dim == 3 else SimConfig2


def cell_list_type(dim: int):
    return CellList3 if dim == 3 else CellList2


class HostParticles:
    """An AoS ``Particle`` array plus the ``ParticleSystem`` header that points at it.

    Keeps the numpy buffer alive for as long as the struct is used.
    """

    def __init__(self, dim: int, pos, vel, types, capacity: int | None = None):
        pos = np.asarray(pos, dtype=np.float64).reshape(-1, dim)
        vel = np.asarray(vel, dtype=np.float64).reshape(-1, dim)
        types = np.asarray(types, dtype=np.int32).reshape(-1)
        n = pos.shape[0]
        cap = max(n, capacity or n, 1)
        self.dim = dim
        self.arr = np.zeros(cap, dtype=particle_dtype(dim))
        self.arr["pos"][:n] = pos
        self.arr["vel"][:n] = vel
        self.arr["type"][:n] = types
        self.ps = ParticleSystem()
        self.ps.particles = self.arr.ctypes.data
        self.ps.num = n
        self.ps.capacity = cap

    @property
    def n(self) -> int:
        return int(self.ps.num)

    @property
    def view(self) -> np.ndarray:
        return self.arr[: self.n]

    def copy(self) -> "HostParticles":
        v = self.view
        h = HostParticles(self.dim, v["pos"], v["vel"], v["type"], capacity=self.arr.shape[0])
        h.arr[: self.n] = v
        h.ps.n0 = self.ps.n0
        h.ps.lambda_ = self.ps.lambda_
        h.ps.C_LL = self.ps.C_LL
        h.ps.C_SL = self.ps.C_SL
        h.ps.n0_count = self.ps.n0_count
        return h


class HostNeighborList:
    """Owns the ``int[num * max_neighbors]`` list of the reference layout."""

    def __init__(self, num: int, max_neighbors: int):
        self.neighbors = np.zeros(max(num, 1) * max_neighbors, dtype=np.int32)
        self.count = np.zeros(max(num, 1), dtype=np.int32)
        self.nl = NeighborList()
        self.nl.neighbors = self.neighbors.ctypes.data_as(C.POINTER(C.c_int))
        self.nl.count = self.count.ctypes.data_as(C.POINTER(C.c_int))
        self.nl.max_neighbors = max_neighbors

    def sets(self, n: int):
        m = self.nl.max_neighbors
        return [self.neighbors[i * m: i * m + self.count[i]] for i in range(n)]
