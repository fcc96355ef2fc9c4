"""ctypes front end of the CPU checker libraries (test infrastructure only).

* ``Oracle(dim)``     -- the C restatement (liboracle3d.so / liboracle2d.so)
* ``Reference(kind)`` -- the reference compiled from its own sources into
  oracle/_ref/ ("3d" = 3-D OpenMP variant, "2d" = 2-D).  The 3-D serial
  variant is not built: its SimConfig carries extra friction fields, and the
  OpenMP variant reproduces it bit for bit (its dot products stay serial).

Both operate on the AoS structs of ``mps_b200.types``.  Only tests,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use this
module.  ``make -C oracle`` builds the libraries.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mps_b200 import types as T

HERE = os.path.dirname(os.path.abspath(__file__))


def build(quiet: bool = True) -> None:
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        build()
    return C.CDLL(path)


P = C.c_void_p
PS = C.POINTER(T.ParticleSystem)
NL = C.POINTER(T.NeighborList)


class Oracle:
    """The C restatement, one library per dimension."""

    def __init__(self, dim: int = 3):
        self.dim = dim
        self.lib = _load(os.path.join(HERE, f"liboracle{dim}d.so"))
        L = self.lib
        CL = C.POINTER(T.cell_list_type(dim))
        CF = C.POINTER(T.sim_config_type(dim))
        self.CL, self.CF = CL, CF
        sig = {
            "oracle_calc_initial_params": (None, [PS, CF]),
            "oracle_calc_initial_params_cells": (None, [PS, CF]),
            "oracle_cell_list_init": (C.c_int, [CL, C.c_int, C.c_double, P, P]),
            "oracle_neighbor_search": (C.c_int, [NL, PS, CL, C.c_double]),
            "oracle_number_density": (None, [PS, NL, CF]),
            "oracle_viscosity": (None, [PS, NL, CF]),
            "oracle_surface_tension": (None, [PS, NL, CF]),
            "oracle_surface_tension_SL": (None, [PS, NL, CF]),
            "oracle_pressure_gradient": (C.c_int, [PS, NL, CF]),
            "oracle_judge_free_surface": (None, [PS, C.c_double]),
            "oracle_neighbor_count": (None, [PS, NL, CF]),
            "oracle_judge_free_surface_by_count": (None, [PS, C.c_double]),
            "oracle_clamp_pressure": (None, [PS]),
            "oracle_collision": (C.c_int, [PS, NL, CF]),
            "oracle_solve_pressure": (C.c_int, [PS, NL, CF]),
            "oracle_assemble_ppe": (C.c_int, [PS, NL, CF, P, P, P, P, P, C.POINTER(C.c_longlong)]),
            "oracle_apply_wall_boundary": (None, [PS]),
            "oracle_remove_out_of_bounds": (None, [PS, CF]),
            "oracle_step": (C.c_int, [PS, NL, CL, CF]),
            "oracle_step_driven": (C.c_int, [PS, NL, CL, CF, P, C.c_double, C.c_double, C.c_int, C.c_int]),
            "oracle_ic0_csr": (C.c_int, [C.c_int, P, P, P, P]),
            "oracle_cell_inverses": (None, [C.c_int, P, P, P, P, P, C.c_int, P]),
            "oracle_ic0_apply_csr": (None, [C.c_int, P, P, P, P, P]),
            "oracle_last_iterations": (C.c_int, []),
            **({"oracle_set_friction": (None, [P]), "oracle_apply_friction": (None, [PS, NL, CF])} if dim == 3 else {}),
            "oracle_last_residual": (C.c_double, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args

    def set_friction(self, cfg) -> None:
        """The friction parameters of the 3-D serial variant (3-D only), from
        the config's attributes (mps_b200.types.FRICTION_DEFAULTS otherwise)."""
        class _F(C.Structure):
            _fields_ = [("enabled", C.c_int), ("delta_theta", C.c_double), ("alpha", C.c_double),
                        ("velocity_threshold", C.c_double)]
        d = T.FRICTION_DEFAULTS
        f = _F(int(getattr(cfg, "friction_enabled", d["friction_enabled"])),
               float(getattr(cfg, "friction_delta_theta", d["friction_delta_theta"])),
               float(getattr(cfg, "dynamic_friction_alpha", d["dynamic_friction_alpha"])),
               float(getattr(cfg, "friction_velocity_threshold", d["friction_velocity_threshold"])))
        self.lib.oracle_set_friction(C.byref(f))

    # --- convenience wrappers -------------------------------------------------
    def ic0_csr(self, rp, ci, v):
        """IC(0) of a CSR matrix in its own numbering; the factor in A's
        pattern (L below, 1/L_ii on, L^T above the diagonal)."""
        rp = np.ascontiguousarray(rp, dtype=np.int32)
        ci = np.ascontiguousarray(ci, dtype=np.int32)
        v = np.ascontiguousarray(v, dtype=np.float64)
        F = np.zeros_like(v)
        if self.lib.oracle_ic0_csr(len(rp) - 1, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, F.ctypes.data):
            raise MemoryError("oracle_ic0_csr")
        return F

    def cell_inverses(self, cells, inv_off, rp, ci, F, max_m=64):
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        inv_off = np.ascontiguousarray(inv_off, dtype=np.int32)
        rp = np.ascontiguousarray(rp, dtype=np.int32)
        ci = np.ascontiguousarray(ci, dtype=np.int32)
        F = np.ascontiguousarray(F, dtype=np.float64)
        inv = np.zeros(max(int(inv_off[-1]), 1))
        self.lib.oracle_cell_inverses(len(cells), cells.ctypes.data, inv_off.ctypes.data, rp.ctypes.data,
                                      ci.ctypes.data, F.ctypes.data, int(max_m), inv.ctypes.data)
        return inv

    def ic0_apply_csr(self, rp, ci, F, r):
        rp = np.ascontiguousarray(rp, dtype=np.int32)
        ci = np.ascontiguousarray(ci, dtype=np.int32)
        F = np.ascontiguousarray(F, dtype=np.float64)
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        self.lib.oracle_ic0_apply_csr(len(rp) - 1, rp.ctypes.data, ci.ctypes.data, F.ctypes.data, r.ctypes.data,
                                      z.ctypes.data)
        return z

    def cell_list(self, num: int, re: float, cfg):
        cl = T.cell_list_type(self.dim)()
        dmin = (C.c_double * self.dim)(*cfg.domain_min)
        dmax = (C.c_double * self.dim)(*cfg.domain_max)
        rc = self.lib.oracle_cell_list_init(C.byref(cl), num, re, C.cast(dmin, P), C.cast(dmax, P))
        if rc != 0:
            raise MemoryError("cell list")
        return cl

    def assemble(self, hp: T.HostParticles, nl: T.HostNeighborList, cfg):
        n = hp.n
        eq = np.zeros(max(n, 1), dtype=np.int32)
        nnz = C.c_longlong(0)
        n_eq = self.lib.oracle_assemble_ppe(C.byref(hp.ps), C.byref(nl.nl), C.byref(cfg),
                                           eq.ctypes.data, None, None, None, None, C.byref(nnz))
        rp = np.zeros(n_eq + 1, dtype=np.int32)
        ci = np.zeros(max(nnz.value, 1), dtype=np.int32)
        va = np.zeros(max(nnz.value, 1), dtype=np.float64)
        b = np.zeros(max(n_eq, 1), dtype=np.float64)
        self.lib.oracle_assemble_ppe(C.byref(hp.ps), C.byref(nl.nl), C.byref(cfg),
                                     eq.ctypes.data, rp.ctypes.data, ci.ctypes.data,
                                     va.ctypes.data, b.ctypes.data, None)
        return eq[:n], rp, ci[: nnz.value], va[: nnz.value], b[:n_eq]

    def initial_params(self, hp: T.HostParticles, cfg, cells: bool = True):
        f = self.lib.oracle_calc_initial_params_cells if cells else self.lib.oracle_calc_initial_params
        f(C.byref(hp.ps), C.byref(cfg))

    def search(self, nl: T.HostNeighborList, hp: T.HostParticles, cl, re: float) -> int:
        return self.lib.oracle_neighbor_search(C.byref(nl.nl), C.byref(hp.ps), C.byref(cl), re)

    def step(self, hp, nl, cl, cfg) -> int:
        return self.lib.oracle_step(C.byref(hp.ps), C.byref(nl.nl), C.byref(cl), C.byref(cfg))

    def step_driven(self, hp, nl, cl, cfg, rest: np.ndarray, amp: float, freq: float, axis: int, step: int) -> int:
        """A step with driven walls (rest: the walls' rest coordinate along
        `axis`, per particle; step: index of the step being taken)."""
        rest = np.ascontiguousarray(rest, dtype=np.float64)
        return self.lib.oracle_step_driven(C.byref(hp.ps), C.byref(nl.nl), C.byref(cl), C.byref(cfg),
                                           rest.ctypes.data, amp, freq, axis, step)


class Reference:
    """The reference's own sources compiled into oracle/_ref/ (see oracle/Makefile).

    Its functions read the global ``SimConfig *g_config``; ``set_config``
    points it at a caller-owned struct, as the reference's main.c does.
    """

    LIBS = {"3d": ("libref3d.so", 3), "2d": ("libref2d.so", 2), "3s": ("libref3s.so", 3)}

    def __init__(self, kind: str = "3d"):
        fname, dim = self.LIBS[kind]
        path = os.path.join(HERE, "_ref", fname)
        if not os.path.exists(path):
            build()
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.kind, self.dim = kind, dim
        self.lib = C.CDLL(path)
        L = self.lib
        CL = C.POINTER(T.cell_list_type(dim))
        self.CL = CL
        sig = {
            "particle_system_calc_initial_params": (None, [PS]),
            "neighbor_search_cell_linked_list": (None, [NL, PS, CL, C.c_double]),
            "calc_particle_number_density": (None, [PS, NL]),
            "calc_viscosity_term": (None, [PS, NL]),
            "calc_pressure_gradient": (None, [PS, NL]),
            "judge_free_surface": (None, [PS, C.c_double]),
            "calc_neighbor_count": (None, [PS, NL]),
            "judge_free_surface_by_count": (None, [PS, C.c_double]),
            "clamp_pressure": (None, [PS]),
            "solve_pressure": (None, [PS, NL]),
            "apply_wall_boundary": (None, [PS]),
            "simulation_step": (None, [PS, NL, CL, C.c_int]),
            "cell_list_create": (CL, [C.c_int, C.c_double, P, P]),
            "cell_list_free": (None, [CL]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L.collision.restype = None
        L.collision.argtypes = [PS, NL] if dim == 3 else [PS]
        L.remove_out_of_bounds.restype = None
        L.remove_out_of_bounds.argtypes = [PS] + [C.c_double] * (2 * dim)
        self._cfg_ref = None

    def set_config(self, cfg) -> None:
        """Point g_config at `cfg`; for the 3-D serial variant ("3s") at a copy
        in its own layout (friction fields from the config's attributes)."""
        if self.kind == "3s":
            cfg = T.serial_config(cfg)
        self._cfg_ref = cfg
        C.c_void_p.in_dll(self.lib, "g_config").value = C.addressof(cfg)

    def cell_list(self, num: int, re: float, cfg):
        dmin = (C.c_double * self.dim)(*cfg.domain_min)
        dmax = (C.c_double * self.dim)(*cfg.domain_max)
        cl = self.lib.cell_list_create(num, re, C.cast(dmin, P), C.cast(dmax, P))
        if not cl:
            raise MemoryError("cell list")
        return cl

    def step(self, hp, nl, cl, step: int = 1) -> None:
        self.lib.simulation_step(C.byref(hp.ps), C.byref(nl.nl), cl, step)
