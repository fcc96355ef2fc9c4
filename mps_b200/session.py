"""Python host side over the C ABI: one device-resident particle system.

Mirrors the reference's driver (``mps_fluid3D_parallel/src/main.c:87-138`` and
``simulation.c:123-181``): load a deck, compute n0/lambda, run the initial
neighbour search, then step.  Arrays cross the boundary as the reference's
AoS ``Particle`` records (``mps_b200.types.particle_dtype``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .types import HostParticles, particle_dtype


class Session:
    def __init__(self, cfg, dim: int, capacity: int, precision: int = _lib.PREC_FP64,
                 refine_tolerance: float = 0.0, params: _lib.MpsParams | None = None):
        self.lib = _lib.load()
        self.dim = dim
        self.cfg = cfg
        self.params = params or _lib.params_from_config(cfg, dim, precision, refine_tolerance)
        h = C.c_void_p()
        self._check(self.lib.mps_session_create(C.byref(h), C.byref(self.params), int(capacity)), h=None)
        self.h = h
        self.n = 0

    # ---- plumbing -----------------------------------------------------------
    def _check(self, rc: int, h="self"):
        if rc != _lib.MPS_OK:
            what = ""
            if h == "self" and getattr(self, "h", None):
                what = (self.lib.mps_last_error(self.h) or b"").decode()
            raise _lib.MpsError(rc, what)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mps_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state --------------------------------------------------------------
    def upload(self, hp: HostParticles):
        self._check(self.lib.mps_upload_particles(self.h, hp.arr.ctypes.data, hp.n))
        self.n = hp.n

    def upload_soa(self, pos, vel, types):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        types = np.ascontiguousarray(types, dtype=np.int32)
        n = types.shape[0]
        self._check(self.lib.mps_upload_soa(self.h, pos.ctypes.data, vel.ctypes.data, types.ctypes.data, n))
        self.n = n

    def download(self, hp: HostParticles | None = None) -> np.ndarray:
        out = np.zeros(self.n, dtype=particle_dtype(self.dim)) if hp is None else hp.arr
        self._check(self.lib.mps_download_particles(self.h, out.ctypes.data, self.n))
        return out[: self.n]

    def pressure(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float64)
        self._check(self.lib.mps_download_pressure(self.h, out.ctypes.data, self.n))
        return out

    # ---- reference quantities ----------------------------------------------------
    def compute_initial_params(self):
        n0, lam, n0c = C.c_double(), C.c_double(), C.c_int()
        self._check(self.lib.mps_compute_initial_params(self.h, C.byref(n0), C.byref(lam), C.byref(n0c)))
        return n0.value, lam.value, n0c.value

    def set_initial_params(self, n0: float, lam: float, n0_count: int = 0):
        self._check(self.lib.mps_set_initial_params(self.h, n0, lam, n0_count))

    def set_precision(self, precision: int):
        """MPS_PREC_FP64 or MPS_PREC_MIXED from the next step on."""
        self._check(self.lib.mps_set_precision(self.h, int(precision)))
        self.params.precision = int(precision)

    # ---- stepping -------------------------------------------------------------
    def neighbor_search(self):
        self._check(self.lib.mps_neighbor_search(self.h))

    def step(self, nsteps: int = 1):
        self._check(self.lib.mps_step(self.h, int(nsteps)))

    def step_with_list(self, neighbors: np.ndarray, count: np.ndarray, max_nb: int):
        neighbors = np.ascontiguousarray(neighbors, dtype=np.int32)
        count = np.ascontiguousarray(count, dtype=np.int32)
        self._check(self.lib.mps_step_with_list(self.h, neighbors.ctypes.data, count.ctypes.data, int(max_nb)))

    def run_stage(self, stage: str, neighbors=None, count=None, max_nb: int = 0, arg: float = 0.0):
        nb = cnt = None
        if neighbors is not None:
            neighbors = np.ascontiguousarray(neighbors, dtype=np.int32)
            count = np.ascontiguousarray(count, dtype=np.int32)
            nb, cnt = neighbors.ctypes.data, count.ctypes.data
        self._check(self.lib.mps_run_stage(self.h, _lib.STAGES[stage], nb, cnt, int(max_nb), float(arg)))

    # ---- introspection ------------------------------------------------------------
    def neighbor_list(self, max_nb: int):
        nb = np.zeros(self.n * max_nb, dtype=np.int32)
        cnt = np.zeros(self.n, dtype=np.int32)
        self._check(self.lib.mps_get_neighbor_list(self.h, nb.ctypes.data, cnt.ctypes.data, int(max_nb)))
        return nb, cnt

    def neighbor_counts(self, max_nb: int):
        cnt = np.zeros(self.n, dtype=np.int32)
        self._check(self.lib.mps_get_neighbor_list(self.h, None, cnt.ctypes.data, int(max_nb)))
        return cnt

    def cell_index(self):
        out = np.zeros(self.n, dtype=np.int32)
        self._check(self.lib.mps_get_cell_index(self.h, out.ctypes.data))
        return out

    def cell_links(self, total_cells: int):
        head = np.zeros(total_cells, dtype=np.int32)
        nxt = np.zeros(self.n, dtype=np.int32)
        self._check(self.lib.mps_get_cell_links(self.h, head.ctypes.data, nxt.ctypes.data, int(total_cells)))
        return head, nxt

    def ppe(self):
        n_eq, nnz = C.c_int(), C.c_longlong()
        self._check(self.lib.mps_get_ppe(self.h, None, None, None, None, None, C.byref(n_eq), C.byref(nnz)))
        eq = np.zeros(self.n, dtype=np.int32)
        rp = np.zeros(n_eq.value + 1, dtype=np.int32)
        ci = np.zeros(max(nnz.value, 1), dtype=np.int32)
        va = np.zeros(max(nnz.value, 1), dtype=np.float64)
        b = np.zeros(max(n_eq.value, 1), dtype=np.float64)
        self._check(self.lib.mps_get_ppe(self.h, eq.ctypes.data, rp.ctypes.data, ci.ctypes.data, va.ctypes.data,
                                         b.ctypes.data, C.byref(n_eq), C.byref(nnz)))
        return eq, rp, ci[: nnz.value], va[: nnz.value], b[: n_eq.value]

    def ic0(self):
        """The last step's PPE and IC(0) factor in the solver's numbering:
        dict of row_ptr, col, A, F, b (numpy)."""
        n_eq, nnz = C.c_int(), C.c_longlong()
        self._check(self.lib.mps_get_ic0(self.h, None, None, None, None, None, C.byref(n_eq), C.byref(nnz)))
        ne, nz = n_eq.value, nnz.value
        rp = np.zeros(ne + 1, dtype=np.int32)
        ci = np.zeros(nz, dtype=np.int32)
        A = np.zeros(nz)
        F = np.zeros(nz)
        b = np.zeros(ne)
        self._check(self.lib.mps_get_ic0(self.h, rp.ctypes.data, ci.ctypes.data, A.ctypes.data, F.ctypes.data,
                                         b.ctypes.data, C.byref(n_eq), C.byref(nnz)))
        return {"row_ptr": rp, "col": ci, "A": A, "F": F, "b": b}

    def cell_blocks(self):
        """(cells (ncells, 2) [first row, unknowns], inv_off, inv, colour_rows)."""
        nc, ninv = C.c_int(), C.c_longlong()
        cr = np.zeros(9, dtype=np.int32)
        self._check(self.lib.mps_get_cell_blocks(self.h, None, None, None, cr.ctypes.data, C.byref(nc),
                                                 C.byref(ninv)))
        cells = np.zeros((nc.value, 2), dtype=np.int32)
        off = np.zeros(nc.value + 1, dtype=np.int32)
        inv = np.zeros(max(ninv.value, 1))
        self._check(self.lib.mps_get_cell_blocks(self.h, cells.ctypes.data, off.ctypes.data, inv.ctypes.data,
                                                 cr.ctypes.data, C.byref(nc), C.byref(ninv)))
        return cells, off, inv, cr[: (1 << self.dim) + 1]

    def apply_preconditioner(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        self._check(self.lib.mps_apply_preconditioner(self.h, r.ctypes.data, z.ctypes.data))
        return z

    def metrics(self) -> dict:
        m = _lib.MpsMetrics()
        self._check(self.lib.mps_get_metrics(self.h, C.byref(m)))
        return {f: getattr(m, f) for f, _ in m._fields_}

    def set_profiling(self, on: bool = True):
        self._check(self.lib.mps_set_profiling(self.h, int(bool(on))))

    def reset_metrics(self):
        self._check(self.lib.mps_reset_metrics(self.h))

    @property
    def stream(self) -> int:
        return int(self.lib.mps_get_stream(self.h) or 0)

    # ---- differentiation form -------------------------------------------------------
    def state_bytes(self) -> int:
        b = C.c_size_t()
        self._check(self.lib.mps_state_bytes(self.h, C.byref(b)))
        return b.value

    def state_save(self, ptr: int):
        """Checkpoint the current state into a host or device buffer of
        state_bytes() bytes at address ``ptr``."""
        self._check(self.lib.mps_state_save(self.h, ptr))

    def state_load(self, ptr: int):
        self._check(self.lib.mps_state_load(self.h, ptr))

    def adjoint_seed(self, lam_pos=None, lam_vel=None):
        """Adjoint of the next reversed step's output, (n, dim) arrays in
        reference order (None = zero); clears the parameter gradients."""
        def arr(a):
            return None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.n, self.dim)
        lx, lu = arr(lam_pos), arr(lam_vel)
        self._check(self.lib.mps_adjoint_seed(self.h, None if lx is None else lx.ctypes.data,
                                              None if lu is None else lu.ctypes.data))

    def adjoint_pressure_seed(self, dLdP=None):
        """dL/dP of the pressures computed by the step that the next
        step_adjoint reverses, (n,) in reference order (None clears)."""
        if dLdP is None:
            self._check(self.lib.mps_adjoint_pressure_seed(self.h, None, self.n))
            return
        a = np.ascontiguousarray(dLdP, dtype=np.float64).reshape(self.n)
        self._check(self.lib.mps_adjoint_pressure_seed(self.h, a.ctypes.data, self.n))

    def step_adjoint(self):
        self._check(self.lib.mps_step_adjoint(self.h))

    def adjoint_get(self):
        """(lam_pos, lam_vel, grad_gravity, grad_viscosity, grad_drive[amp, freq])."""
        lx = np.zeros((self.n, self.dim), dtype=np.float64)
        lu = np.zeros((self.n, self.dim), dtype=np.float64)
        gg = np.zeros(self.dim, dtype=np.float64)
        gd = np.zeros(2, dtype=np.float64)
        gn = C.c_double()
        self._check(self.lib.mps_adjoint_get(self.h, lx.ctypes.data, lu.ctypes.data, gg.ctypes.data,
                                             C.byref(gn), gd.ctypes.data))
        return lx, lu, gg, gn.value, gd

    def set_wall_drive(self, amp: float, freq: float, axis: int = 0):
        """Driven walls (mps_params_t.wall_drive_*); amp = 0 is the reference's fixed walls."""
        self.params.wall_drive_amp = float(amp)
        self.params.wall_drive_freq = float(freq)
        self.params.wall_drive_axis = int(axis)
        self._check(self.lib.mps_update_params(self.h, C.byref(self.params)))


def start(cfg, dim: int, hp: HostParticles, capacity: int | None = None, **kw) -> Session:
    """Upload, compute n0/lambda on the device, run the initial neighbour search."""
    s = Session(cfg, dim, capacity or hp.n, **kw)
    s.upload(hp)
    n0, lam, n0c = s.compute_initial_params()
    hp.ps.n0, hp.ps.lambda_, hp.ps.n0_count = n0, lam, n0c
    s.neighbor_search()
    return s
