"""ctypes binding of ``libmps_b200.so`` (the C ABI in ``include/mps_b200.h``).

The library is built in-tree by ``mps_b200.build`` (``__graft_entry__.build()``).
There is no fallback: importing a session without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmps_b200.so")

MPS_OK = 0
ERRORS = {
    -1: "MPS_ERR_INVALID",
    -2: "MPS_ERR_CUDA",
    -3: "MPS_ERR_OOM",
    -4: "MPS_ERR_NEIGHBOR_OVERFLOW",
    -5: "MPS_ERR_UNSUPPORTED",
    -6: "MPS_ERR_NOT_CONVERGED",
    -7: "MPS_ERR_NAN",
}
PREC_FP64, PREC_MIXED = 0, 1

STAGES = {
    "density": 1,
    "viscosity": 2,
    "gradient": 3,
    "neighbor_count": 4,
    "collision": 5,
    "solve_pressure": 6,
    "surface": 7,
    "clamp": 8,
    "wall": 9,
    "out_of_bounds": 10,
    "surface_by_count": 11,
    "surface_tension": 12,
    "surface_tension_sl": 13,
}


class MpsParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("particle_distance", C.c_double),
        ("influence_radius_lap", C.c_double),
        ("influence_radius_n", C.c_double),
        ("max_neighbors", C.c_int),
        ("wall_layers", C.c_int),
        ("density", C.c_double),
        ("viscosity", C.c_double),
        ("gravity", C.c_double * 3),
        ("dt", C.c_double),
        ("solver_type", C.c_int),
        ("cg_max_iter", C.c_int),
        ("cg_tolerance", C.c_double),
        ("relaxation_coeff", C.c_double),
        ("clamp_negative_pressure", C.c_int),
        ("ppe_type", C.c_int),
        ("c_ppe", C.c_double),
        ("gamma_ppe", C.c_double),
        ("surface_threshold", C.c_double),
        ("surface_detection_method", C.c_int),
        ("surface_count_threshold", C.c_double),
        ("restitution_coeff", C.c_double),
        ("collision_distance_ratio", C.c_double),
        ("surface_tension_enabled", C.c_int),
        ("domain_min", C.c_double * 3),
        ("domain_max", C.c_double * 3),
        ("cmps_gradient", C.c_int),
        ("use_analytical_lambda", C.c_int),
        ("hs_mode", C.c_int),
        ("precision", C.c_int),
        ("refine_tolerance", C.c_double),
        ("wall_drive_amp", C.c_double),
        ("wall_drive_freq", C.c_double),
        ("wall_drive_axis", C.c_int),
        ("influence_radius_st", C.c_double),
        ("surface_tension_coeff", C.c_double),
        ("wetting_angle_SL", C.c_double),
        ("friction_enabled", C.c_int),
        ("friction_delta_theta", C.c_double),
        ("dynamic_friction_alpha", C.c_double),
        ("friction_velocity_threshold", C.c_double),
    ]


class MpsGrid(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("origin", C.c_double * 3),
        ("cell_size", C.c_double),
        ("dims", C.c_int * 3),
    ]


class MpsMetrics(C.Structure):
    _fields_ = [
        ("ppe_iterations", C.c_int),
        ("ppe_outer", C.c_int),
        ("ppe_residual", C.c_double),
        ("n_eq", C.c_int),
        ("nnz", C.c_longlong),
        ("n_fluid", C.c_int),
        ("n_ghost", C.c_int),
        ("converged", C.c_int),
        ("total_iterations", C.c_longlong),
        ("total_steps", C.c_longlong),
        ("ms_ops", C.c_double),
        ("ms_assembly", C.c_double),
        ("ms_factor", C.c_double),
        ("ms_solve", C.c_double),
        ("prof_spmv_ms", C.c_double),
        ("prof_spmv_launches", C.c_longlong),
        ("prof_fwd_ms", C.c_double),
        ("prof_fwd_sweeps", C.c_longlong),
        ("prof_bwd_ms", C.c_double),
        ("prof_bwd_sweeps", C.c_longlong),
        ("prof_vec_ms", C.c_double),
        ("prof_iterations", C.c_longlong),
        ("prof_nnz_sum", C.c_longlong),
        ("prof_rows_sum", C.c_longlong),
        ("ppe_true_residual", C.c_double),
        ("ppe_bnorm", C.c_double),
        ("ppe_rounding_floor", C.c_double),
        ("sweep_cross_lo", C.c_longlong),
        ("sweep_cross_up", C.c_longlong),
        ("sweep_inverse_entries", C.c_longlong),
        ("prof_pcg_ms", C.c_double),
        ("prof_pcg_launches", C.c_longlong),
        ("prof_pcg_iterations", C.c_longlong),
    ]


# Every symbol include/mps_b200.h declares, with its ctypes signature.
P = C.c_void_p
I = C.c_int
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)
SIGNATURES = {
    "mps_version": (I, []),
    "mps_error_string": (C.c_char_p, [I]),
    "mps_session_create": (I, [C.POINTER(P), C.POINTER(MpsParams), I]),
    "mps_session_destroy": (I, [P]),
    "mps_update_params": (I, [P, C.POINTER(MpsParams)]),
    "mps_set_precision": (I, [P, I]),
    "mps_last_error": (C.c_char_p, [P]),
    "mps_upload_particles": (I, [P, P, I]),
    "mps_download_particles": (I, [P, P, I]),
    "mps_upload_soa": (I, [P, P, P, P, I]),
    "mps_download_pressure": (I, [P, P, I]),
    "mps_compute_initial_params": (I, [P, DP, DP, IP]),
    "mps_set_initial_params": (I, [P, C.c_double, C.c_double, I]),
    "mps_neighbor_search": (I, [P]),
    "mps_step": (I, [P, I]),
    "mps_step_with_list": (I, [P, P, P, I]),
    "mps_get_neighbor_list": (I, [P, P, P, I]),
    "mps_get_cell_index": (I, [P, P]),
    "mps_get_cell_links": (I, [P, P, P, I]),
    "mps_get_ppe": (I, [P, P, P, P, P, P, IP, C.POINTER(C.c_longlong)]),
    "mps_get_ic0": (I, [P, P, P, P, P, P, IP, C.POINTER(C.c_longlong)]),
    "mps_get_cell_blocks": (I, [P, P, P, P, P, IP, C.POINTER(C.c_longlong)]),
    "mps_apply_preconditioner": (I, [P, P, P]),
    "mps_get_metrics": (I, [P, C.POINTER(MpsMetrics)]),
    "mps_get_stream": (P, [P]),
    "mps_launch_count": (C.c_ulonglong, []),
    "mps_surface_tension_coeffs": (I, [C.POINTER(MpsParams), DP, DP]),
    "mps_set_profiling": (I, [P, I]),
    "mps_reset_metrics": (I, [P]),
    "mps_run_stage": (I, [P, I, P, P, I, C.c_double]),
    "mps_cell_sort_noalloc": (I, [C.POINTER(MpsGrid), P, P, I, P, P, P, P]),
    "mps_state_bytes": (I, [P, C.POINTER(C.c_size_t)]),
    "mps_state_save": (I, [P, P]),
    "mps_state_load": (I, [P, P]),
    "mps_adjoint_seed": (I, [P, P, P]),
    "mps_adjoint_pressure_seed": (I, [P, P, I]),
    "mps_step_adjoint": (I, [P]),
    "mps_adjoint_get": (I, [P, P, P, P, P, P]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()')"
        )
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class MpsError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{ERRORS.get(code, code)}: {what}")


def params_from_config(cfg, dim: int, precision: int = PREC_FP64, refine_tolerance: float = 0.0) -> MpsParams:
    """The session parameters of a reference ``SimConfig`` (already parsed)."""
    p = MpsParams()
    p.dim = dim
    for f in ("particle_distance", "influence_radius_lap", "influence_radius_n", "max_neighbors",
              "wall_layers", "density", "viscosity", "dt", "solver_type", "cg_max_iter", "cg_tolerance",
              "relaxation_coeff", "clamp_negative_pressure", "ppe_type", "c_ppe", "gamma_ppe",
              "surface_threshold", "surface_detection_method", "surface_count_threshold",
              "restitution_coeff", "collision_distance_ratio", "surface_tension_enabled",
              "cmps_gradient", "use_analytical_lambda", "hs_mode", "influence_radius_st",
              "surface_tension_coeff", "wetting_angle_SL"):
        setattr(p, f, getattr(cfg, f))
    for d in range(dim):
        p.gravity[d] = cfg.gravity[d]
        p.domain_min[d] = cfg.domain_min[d]
        p.domain_max[d] = cfg.domain_max[d]
    from .types import FRICTION_DEFAULTS
    for f, v in FRICTION_DEFAULTS.items():   # 3-D serial-variant keys, config attributes when parsed
        setattr(p, f, getattr(cfg, f, v))
    p.precision = precision
    p.refine_tolerance = refine_tolerance
    return p
