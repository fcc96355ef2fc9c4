"""Throughput of the MPS time step on B200: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c1] [--precision fp64]

A step is one full MPS time step (simulation.c:19-118 of the reference) of
the 3-D dam break named by --workload, device-resident: explicit viscosity
and collision, the cell-sort neighbour search, number density and surface
flags, PPE assembly, IC(0) factorisation and the PCG solve to the absolute
tolerance 1e-9, the pressure gradient and the correction.  `value` is fluid
particle-steps/s over all ranks (each rank runs an independent replica with
its own seed: the time step has no partition that avoids a halo exchange
per operator and changes the IC(0) preconditioner).  The workload's PPE
matrix alone is ~1.5 GB, far above the 126 MB L2, so consecutive steps do
not run from cache.

Other keys: `roofline` for the dominant kernel (the CG SpMV, timed with CUDA
events on the library's stream during the timed steps), `cpu_baseline` (the
reference compiled from source, OpenMP on all host cores, on a bounded
sample of the same workload), `e2e` (the same metric through the C ABI with
host buffers copied in and out every step), `clocks` (nvidia-smi sampled
during the timed region), `gpu_launches` (kernels this library launched in
the timed region), `adjoint` (N=1: cost of the differentiation form on the
same workload -- a short rollout's backward per step against its forward
per step, and one isolated mps_step_adjoint).

--impl reference times the reference's own CPU implementation (oracle/_ref)
on the bounded sample, rank 0 only.

--sloshing-adjoint STEPS prints, instead, the differentiation form's cost on
the 3-D sloshing tank with driven walls.

--error-growth STEPS prints, instead, the mixed form's long-run accuracy:
its error growth against the FP64 path next to that of a reordered FP64
run, and integral observables of the three runs (rank 0, one GPU).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D dam-break particle-steps/s: mixed vs FP64 GPU @ p err≤1e-4; adjoint/fwd cost"
UNIT = "fluid particle-steps/s"

WORKLOADS = {
    "c1": "3-D dam break, tank 1.6x0.6x0.6 m, column 0.4x0.6x0.3 m, l0=0.005 m, "
          "1,170,276 particles (576,000 fluid), dt 5e-4, ICCG tol 1e-9",
    "c2": "3-D dam break, tank 1.6x0.6x0.6 m, column 0.4x0.6x0.3 m, l0=0.0035 m, dt 3.5e-4, ICCG tol 1e-9",
}
# The CPU sample: the same dam break at l0 = 0.01 (225,236 particles,
# 72,000 fluid); one reference step there is a few seconds on 8 cores,
# against ~80 s at l0 = 0.005.
CPU_SAMPLE_L0 = 0.01


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# CPU: the reference compiled from source (oracle/_ref), bounded sample
# ---------------------------------------------------------------------------

def reference_cpu_steps(steps: int, warmup: int, l0: float = CPU_SAMPLE_L0, seed: int = 0):
    """Times `steps` reference simulation_step calls (after `warmup` untimed
    ones) on the sample; returns (fluid particle-steps/s, seconds/step, meta)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(host_cores()))
    from mps_b200 import config as CF
    from mps_b200 import types as T
    from mps_b200 import workloads as W
    from oracle.pyoracle import Oracle, Reference

    wl = W.dambreak("c1", l0=l0, seed=seed)
    cfg = wl.config()
    kind = "reference"
    ref = Reference("3d")
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    # n0 / lambda with the oracle's cell-list form of particle.c:69-221 (bit-identical
    # to the reference's O(N^2) loop, which alone would take minutes here)
    Oracle(3).initial_params(hp, cfg)
    ref.set_config(cfg)
    re = CF.neighbor_radius(cfg)
    nl = T.HostNeighborList(hp.n, cfg.max_neighbors)
    cl = ref.cell_list(hp.n, re, cfg)
    ref.lib.neighbor_search_cell_linked_list(C.byref(nl.nl), C.byref(hp.ps), cl, re)
    for s in range(warmup):
        ref.step(hp, nl, cl, s + 1)
    t0 = time.perf_counter()
    for s in range(steps):
        ref.step(hp, nl, cl, warmup + s + 1)
    dt = time.perf_counter() - t0
    ref.lib.cell_list_free(cl)
    meta = {"kind": kind, "cores": int(os.environ["OMP_NUM_THREADS"]),
            "sample": f"c1 geometry at l0={l0} ({wl.n} particles, {wl.n_fluid} fluid), "
                      f"{steps} reference simulation_step call(s) after {warmup} warm-up, "
                      "OpenMP build of mps_fluid3D_parallel compiled from source"}
    return wl.n_fluid * steps / dt, dt / max(steps, 1), meta


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# roofline of the dominant kernel
# ---------------------------------------------------------------------------

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0}, "fallback"


def ncu_traffic(kernel: str):
    """(DRAM bytes per launch, algorithmic bytes per launch) of `kernel` from
    the committed ncu summary (profiles/*.md lines
    'traffic_per_launch_bytes <kernel> <dram bytes> <algorithmic bytes>');
    None when absent.  The bench scales the ratio to its own workload."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for name in sorted(os.listdir(d)):
        if not name.endswith(".md"):
            continue
        for line in open(os.path.join(d, name)):
            t = line.strip().strip("`").split()
            if len(t) == 4 and t[0] == "traffic_per_launch_bytes" and t[1] == kernel:
                return float(t[2]), float(t[3])
    return None


# ---------------------------------------------------------------------------
# the B200 arm
# ---------------------------------------------------------------------------

def max_over_ranks(x: float, dist, device) -> float:
    """The job's time: the maximum of a per-rank time over all ranks (one
    independent replica per rank, so the job ends with its slowest rank)."""
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(n_fluid_per_rank: int, world: int, steps: int, seconds: float) -> float:
    """Fluid particle-steps per second of all replicas together."""
    return n_fluid_per_rank * world * steps / seconds


def run_b200(args, rank: int, world: int, local_rank: int):
    import numpy as np
    import torch

    from mps_b200 import _lib
    from mps_b200 import types as T
    from mps_b200 import workloads as W
    from mps_b200.session import Session

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    wl = W.dambreak(args.workload, seed=1000 + rank, l0=args.l0)
    cfg = wl.config()
    prec = _lib.PREC_MIXED if args.precision == "mixed" else _lib.PREC_FP64
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    sess = Session(cfg, 3, hp.n, precision=prec)
    sess.upload(hp)
    n0, lam, _ = sess.compute_initial_params()
    sess.neighbor_search()
    for _ in range(args.warmup):
        sess.step(1)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(sess.stream)
    sess.reset_metrics()
    clocks = ClockSampler(local_rank) if rank == 0 else None
    lib = _lib.load()

    def barrier():
        if dist is not None:
            dist.barrier()

    # timed region: K steps, no per-kernel events
    barrier()
    torch.cuda.synchronize()
    l0 = lib.mps_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sess.step(1)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = lib.mps_launch_count() - l0
    ms = e0.elapsed_time(e1)
    clk = clocks.stop() if clocks else None
    met = sess.metrics()
    # kernel breakdown: the next min(K, 2) steps again with CUDA events
    # around every CG-loop kernel group (they add a little time, so these
    # steps are not part of `value`)
    sess.reset_metrics()
    sess.set_profiling(True)
    for _ in range(min(args.steps, 2)):
        sess.step(1)
    torch.cuda.synchronize()
    pmet = sess.metrics()
    sess.set_profiling(False)

    ms_max = max_over_ranks(ms, dist, "cuda")
    value = whole_job_value(wl.n_fluid, world, args.steps, ms_max / 1e3)
    iters = met["total_iterations"]

    sess.close()
    e2e = None if args.no_e2e else run_e2e(wl, cfg, args, torch, dist)
    adjoint = None
    if world == 1 and not args.no_adjoint:
        adjoint = run_adjoint_cost(wl, cfg, prec, torch)

    result = None
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        nnz_mean = pmet["prof_nnz_sum"] / max(pmet["prof_iterations"], 1)
        rows_mean = pmet["prof_rows_sum"] / max(pmet["prof_iterations"], 1)
        # SpMV algorithmic bytes per launch: A value + column 4 B per nonzero,
        # row pointer 4 B, p and Ap per row (values 8 B in FP64, 4 B in the
        # mixed form's FP32 inner solve).
        vb = 8.0 if prec == _lib.PREC_FP64 else 4.0
        alg_bytes = (vb + 4.0) * nnz_mean + (4.0 + 2.0 * vb) * rows_mean
        spmv_ms = pmet["prof_spmv_ms"] / max(pmet["prof_spmv_launches"], 1)
        achieved = alg_bytes / (spmv_ms / 1e3) / 1e9
        peak = float(peaks.get("hbm_gbs", 6650.0))
        tr = ncu_traffic("k_cg_spmv")
        traffic = None
        if tr is not None:
            traffic = tr[0] / tr[1] * alg_bytes
        fwd_ms = pmet["prof_fwd_ms"] / max(pmet["prof_fwd_sweeps"], 1)
        bwd_ms = pmet["prof_bwd_ms"] / max(pmet["prof_bwd_sweeps"], 1)
        cpu = None
        if world == 1 and not args.no_cpu:
            v, sec, meta = reference_cpu_steps(args.cpu_steps, 0)
            cpu = {"value": v, "unit": UNIT, "cores": meta["cores"], "kind": meta["kind"], "sample": meta["sample"],
                   "seconds_per_step": sec}
        result = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if prec == _lib.PREC_FP64 else "f32+f64",
            "data": "synthetic",
            "config": {
                "workload": WORKLOADS.get(args.workload, args.workload),
                "particles_per_gpu": wl.n,
                "fluid_per_gpu": wl.n_fluid,
                "precision": args.precision,
                "parallelism": f"replicas x{world}",
                "l2": "inputs larger than L2 (PPE matrix ~1.5 GB per replica)",
                "n0": n0,
                "lambda": lam,
            },
            "total_particle_steps_per_s": wl.n * world * args.steps / (ms_max / 1e3),
            "ppe_iterations_per_step": iters / args.steps,
            "ppe_iterations_per_s": iters / (ms_max / 1e3),
            "stage_ms_last_step": {"ops": met["ms_ops"], "assembly": met["ms_assembly"],
                                   "factor": met["ms_factor"], "solve": met["ms_solve"]},
            "kernel_ms_per_launch": {"k_cg_spmv": spmv_ms, "ic0_forward_sweep(8 colours)": fwd_ms,
                                     "ic0_backward_sweep(8 colours)": bwd_ms,
                                     "cg_vector_kernels_per_iter": pmet["prof_vec_ms"] / max(pmet["prof_iterations"], 1)},
            "roofline": {"kernel": "k_cg_spmv", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "timing": "CUDA events around every SpMV launch on the library stream, over "
                                   "min(steps, 2) further steps right after the timed region",
                         "algorithmic_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "adjoint": adjoint,
            "gpu_launches": int(launches),
            "clocks": clk,
        }
    if dist is not None:
        dist.destroy_process_group()
    return result


def run_adjoint_cost(wl, cfg, prec, torch, steps: int = 2):
    """Cost of the differentiation form on the same workload: a `steps`-step
    rollout (checkpoint at its first step) forward, then its backward
    (segment recompute from the checkpoint + one mps_step_adjoint per step,
    each recomputing its step and reversing it), timed with CUDA events on
    the library's stream after one untimed warm-up rollout; plus one
    isolated state_load + mps_step_adjoint, and the device memory in use at
    the end."""
    import numpy as np

    from mps_b200.adjoint import Rollout

    roll = Rollout(cfg, 3, wl.pos, wl.types, steps, every=steps, precision=prec)
    # one untimed forward and backward: first-use device allocations
    xw, uw, tw = roll.forward(wl.vel, 1.0, cfg.viscosity)
    roll.backward(np.zeros_like(xw), np.zeros_like(uw))
    stream = torch.cuda.ExternalStream(roll.sess.stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    roll._set_params(1.0, cfg.viscosity)
    roll._upload(wl.vel)
    roll.sess.set_initial_params(roll.n0, roll.lam, roll.n0_count)
    roll.sess.neighbor_search()
    torch.cuda.synchronize()
    ev[0].record(stream)
    roll.ckpts = [roll._save()]
    for _ in range(steps):
        roll.sess.step(1)
    ev[1].record(stream)
    torch.cuda.synchronize()
    x, u, t = roll._final()
    fl = (t == 0)[:, None]
    target = wl.pos + 0.001
    lam = 2.0 * (x - target) * fl / max(int(fl.sum()), 1)
    ev[2].record(stream)
    roll.backward(lam, np.zeros_like(u))
    ev[3].record(stream)
    torch.cuda.synchronize()
    roll.sess.state_load(roll.ckpts[0].data_ptr())
    ev[4].record(stream)
    roll.sess.step_adjoint()
    ev[5].record(stream)
    torch.cuda.synchronize()
    free, total = torch.cuda.mem_get_info()
    fwd = ev[0].elapsed_time(ev[1]) / steps
    bwd = ev[2].elapsed_time(ev[3]) / steps
    one = ev[4].elapsed_time(ev[5])
    roll.close()
    return {"workload": "as config.workload", "rollout_steps": steps, "checkpoint_every": steps,
            "fwd_ms_per_step": fwd, "backward_ms_per_step": bwd, "adjoint_over_fwd": bwd / fwd,
            "step_adjoint_ms": one, "step_adjoint_over_fwd": one / fwd,
            "device_memory_in_use_gb": (total - free) / 1e9,
            "note": "backward = segment recompute + per-step recompute and reverse pass incl. the adjoint "
                    "PPE solve; loss = mean squared distance of fluid positions to a shifted target"}


def run_e2e(wl, cfg, args, torch, dist):
    """The same metric through the reference-facing C ABI with host buffers:
    the drop-in simulation_step(ps, nl, cl, step) of libmps3d.so, whose
    particles (AoS) and neighbour list live in pinned host memory.  Every
    call copies the particles and the previous step's list to the device and
    the new particles, list and cell chains back; the drop-in runs the
    line's precision form (mps_dropin_set_precision).  Timed with CUDA events
    around the synchronous calls, max over ranks."""
    import numpy as np

    from mps_b200 import _lib
    from mps_b200 import config as CF
    from mps_b200 import types as T

    lib = C.CDLL(os.path.join(ROOT, "mps_b200", "libmps3d.so"))
    lib.mps_dropin_set_exit_on_error(0)
    # the drop-in runs the same precision form as the timed steps
    prec = _lib.PREC_MIXED if args.precision == "mixed" else _lib.PREC_FP64
    if lib.mps_dropin_set_precision(prec) != 0:
        return None
    PS = C.POINTER(T.ParticleSystem)
    NL = C.POINTER(T.NeighborList)
    CLP = C.POINTER(T.CellList3)
    lib.particle_system_calc_initial_params.argtypes = [PS]
    lib.neighbor_search_cell_linked_list.argtypes = [NL, PS, CLP, C.c_double]
    lib.simulation_step.argtypes = [PS, NL, CLP, C.c_int]
    lib.cell_list_create.restype = CLP
    lib.cell_list_create.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    lib.mps_dropin_last_status.restype = C.c_int
    lib.mps_dropin_release.argtypes = [PS]
    C.c_void_p.in_dll(lib, "g_config").value = C.addressof(cfg)

    n, m = wl.n, cfg.max_neighbors
    dt_p = T.particle_dtype(3)
    p_buf = torch.empty(n * dt_p.itemsize, dtype=torch.uint8, pin_memory=True)
    parts = np.frombuffer(p_buf.numpy(), dtype=dt_p, count=n)
    parts[:] = 0
    parts["pos"] = wl.pos
    parts["vel"] = wl.vel
    parts["type"] = wl.types
    ps = T.ParticleSystem()
    ps.particles = parts.ctypes.data
    ps.num = ps.capacity = n
    nb_buf = torch.empty(n * m, dtype=torch.int32, pin_memory=True)
    cnt_buf = torch.zeros(n, dtype=torch.int32, pin_memory=True)
    nl = T.NeighborList()
    nl.neighbors = C.cast(nb_buf.data_ptr(), C.POINTER(C.c_int))
    nl.count = C.cast(cnt_buf.data_ptr(), C.POINTER(C.c_int))
    nl.max_neighbors = m
    re = CF.neighbor_radius(cfg)
    dmin = (C.c_double * 3)(*cfg.domain_min)
    dmax = (C.c_double * 3)(*cfg.domain_max)
    cl = lib.cell_list_create(n, re, C.cast(dmin, C.c_void_p), C.cast(dmax, C.c_void_p))
    lib.particle_system_calc_initial_params(C.byref(ps))
    lib.neighbor_search_cell_linked_list(C.byref(nl), C.byref(ps), cl, re)
    if lib.mps_dropin_last_status() != 0:
        return None
    cnt = cnt_buf.numpy()
    lib.simulation_step(C.byref(ps), C.byref(nl), cl, 1)           # warm-up call
    steps = args.steps
    h2d = d2h = 0
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    # the drop-in calls are synchronous (host copies in and out), so CUDA
    # events on the idle current stream, after a device synchronize, bracket
    # exactly the loop
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for k in range(steps):
        mc_in = int(cnt.max())
        lib.simulation_step(C.byref(ps), C.byref(nl), cl, 2 + k)
        mc_out = int(cnt.max())
        # bytes copied by the call: AoS particles and the counts both ways,
        # the used columns of the list (pitched copy), the cell chains back
        h2d += n * dt_p.itemsize + 4 * n + 4 * n * mc_in
        d2h += n * dt_p.itemsize + 4 * n + 4 * n * mc_out + 4 * cl.contents.total_cells + 4 * n
    torch.cuda.synchronize()
    ev1.record()
    torch.cuda.synchronize()
    wall = ev0.elapsed_time(ev1) / 1e3
    ok = lib.mps_dropin_last_status() == 0
    lib.mps_dropin_release(C.byref(ps))
    wall = max_over_ranks(wall, dist, "cuda")
    if not ok:
        return None
    world = dist.get_world_size() if dist is not None else 1
    return {"value": whole_job_value(wl.n_fluid, world, steps, wall), "unit": UNIT,
            "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps,
            "ms_per_step": wall / steps * 1e3,
            "call": "simulation_step(ps, nl, cl, step) of libmps3d.so, pinned host AoS + NeighborList",
            "precision": args.precision}


# ---- accuracy of the mixed form over a long run ---------------------------------
#
# A pointwise comparison of two dam-break runs whose reductions differ stops
# being meaningful after a few hundred steps (the flow amplifies rounding
# differences), so the mixed form is reported three ways: its error growth
# against the FP64 path, next to the growth between two FP64 runs that
# differ only in the SpMV's summation order (the reordering noise floor), and
# integral observables of the three runs at the end (fluid count, surge
# front, pressure binned on a fixed grid and time-averaged, a wall-probe
# pressure series).

FLUID_T, WALL_T = 0, 1


def _rel_l2(a, b):
    import numpy as np
    d = float(np.linalg.norm(np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64)))
    nb = float(np.linalg.norm(np.asarray(b, dtype=np.float64)))
    return d / nb if nb > 0 else d


def state_errors(a, ref):
    """Relative L2 differences of one state against a reference state (both
    particle records in reference order): pressure over all particles,
    velocity and position over the particles that are fluid in both, and the
    counts of differing surface flags and types."""
    import numpy as np
    both = (a["type"] == FLUID_T) & (ref["type"] == FLUID_T)
    return {"p_rel": _rel_l2(a["pressure"], ref["pressure"]),
            "v_rel": _rel_l2(a["vel"][both], ref["vel"][both]),
            "x_rel": _rel_l2(a["pos"][both], ref["pos"][both]),
            "surface_flags_differing": int(np.count_nonzero(a["on_surface"] != ref["on_surface"])),
            "types_differing": int(np.count_nonzero(a["type"] != ref["type"]))}


def grid_pressure(state, l0: float, domain, bin_l0: float = 4.0):
    """Mean fluid pressure per cell of a fixed grid of side bin_l0 * l0 over
    the tank (x, y, z >= 0 up to `domain`); returns (sum, count) arrays."""
    import numpy as np
    h = bin_l0 * l0
    dims = [max(1, int(np.ceil(domain[d] / h))) for d in range(3)]
    f = state["type"] == FLUID_T
    x = state["pos"][f]
    idx = [np.clip(np.floor(x[:, d] / h).astype(np.int64), 0, dims[d] - 1) for d in range(3)]
    lin = (idx[0] * dims[1] + idx[1]) * dims[2] + idx[2]
    tot = dims[0] * dims[1] * dims[2]
    ssum = np.bincount(lin, weights=state["pressure"][f], minlength=tot)
    cnt = np.bincount(lin, minlength=tot).astype(np.float64)
    return ssum, cnt


def probe_mask(pos0, types, l0: float, domain, height: float = 0.05, zc: float = 0.15, radius_l0: float = 3.0):
    """The wall probe: particles of the first wall layer behind the +x wall
    (x in (Lx, Lx + 1.5 l0)) within radius_l0 * l0 of (height, zc) in the
    wall's plane (y vertical)."""
    import numpy as np
    lx = domain[0]
    r2 = (pos0[:, 1] - height) ** 2 + (pos0[:, 2] - zc) ** 2
    return (types == WALL_T) & (pos0[:, 0] > lx) & (pos0[:, 0] < lx + 1.5 * l0) & (r2 <= (radius_l0 * l0) ** 2)


def observables(state, probe):
    """Fluid count, surge front (largest x of a fluid particle) and the mean
    pressure over the probe particles."""
    import numpy as np
    f = state["type"] == FLUID_T
    return {"fluid": int(np.count_nonzero(f)),
            "front_x": float(state["pos"][f, 0].max()) if f.any() else 0.0,
            "probe_p": float(state["pressure"][probe].mean()) if probe.any() else 0.0}


def run_error_growth(args):
    """Mixed form and a reordered FP64 run against the FP64 path over
    `args.error_growth` steps of the dam break (workload and l0 as given,
    l0 = 0.01 by default), from the same initial state, in lockstep on one
    GPU.  Prints one JSON line."""
    import numpy as np
    import torch

    from mps_b200 import _lib
    from mps_b200 import types as T
    from mps_b200 import workloads as W
    from mps_b200.session import Session

    steps = int(args.error_growth)
    l0 = args.l0 if args.l0 is not None else 0.01
    wl = W.dambreak(args.workload, seed=1000, l0=l0)
    cfg = wl.config()
    domain = [cfg.domain_max[d] for d in range(3)]
    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)

    def make(prec, lpr):
        old = os.environ.pop("MPS_SPMV_LPR", None)
        if lpr:
            os.environ["MPS_SPMV_LPR"] = str(lpr)
        try:
            s = Session(cfg, 3, hp.n, precision=prec)
        finally:
            os.environ.pop("MPS_SPMV_LPR", None)
            if old is not None:
                os.environ["MPS_SPMV_LPR"] = old
        s.upload(hp)
        return s

    runs = {"fp64": make(_lib.PREC_FP64, 8), "mixed": make(_lib.PREC_MIXED, 0),
            "fp64_reordered": make(_lib.PREC_FP64, 16)}
    n0, lam, nc = runs["fp64"].compute_initial_params()
    for s in runs.values():
        s.set_initial_params(n0, lam, nc)
        s.neighbor_search()
    probe = probe_mask(wl.pos, wl.types, l0, domain)
    marks = sorted({k for k in (1, 10, 50, 100, 200, 300, 400, 500, 600, 700, 800, 900, 1000) if k <= steps} | {steps})
    growth = {k: {key: [] for key in ("p_rel", "v_rel", "x_rel", "surface_flags_differing", "types_differing")}
              for k in ("mixed", "fp64_reordered")}
    obs = {k: [] for k in runs}
    gsum = {k: None for k in runs}
    gcnt = {k: None for k in runs}
    done = 0
    t0 = time.time()
    for mk in marks:
        st = {}
        for k, s in runs.items():
            s.step(mk - done)
            st[k] = s.download().copy()
        torch.cuda.synchronize()
        done = mk
        for k in growth:
            e = state_errors(st[k], st["fp64"])
            for key, v in e.items():
                growth[k][key].append(v)
        for k in runs:
            obs[k].append(observables(st[k], probe))
            if mk >= steps / 2:
                a, c = grid_pressure(st[k], l0, domain)
                gsum[k] = a if gsum[k] is None else gsum[k] + a
                gcnt[k] = c if gcnt[k] is None else gcnt[k] + c
    wall = time.time() - t0
    for s in runs.values():
        s.close()
    occ = np.ones_like(gcnt["fp64"], dtype=bool)
    for k in runs:
        occ &= gcnt[k] > 0
    gmean = {k: gsum[k][occ] / gcnt[k][occ] for k in runs}
    series = {k: np.array([o["probe_p"] for o in obs[k]]) for k in runs}
    final = {k: obs[k][-1] for k in runs}
    return {
        "metric": "mixed-form error growth vs FP64 (with the FP64 reordering noise floor)",
        "workload": wl.name, "particles": int(wl.n), "fluid": int(wl.n_fluid), "steps": steps, "dt": cfg.dt,
        "checkpoints": marks, "growth": growth,
        "final_observables": final,
        "grid_pressure_time_mean_rel_l2": {k: _rel_l2(gmean[k], gmean["fp64"]) for k in ("mixed", "fp64_reordered")},
        "grid": {"bin": "4 l0", "cells_compared": int(occ.sum()),
                 "samples": "checkpoints at or after half the run"},
        "probe": {"particles": int(probe.sum()), "where": "+x wall, y = 0.05 m, z = 0.15 m, radius 3 l0",
                  "series_fp64": [float(v) for v in series["fp64"]],
                  "series_rel_l2": {k: _rel_l2(series[k], series["fp64"]) for k in ("mixed", "fp64_reordered")}},
        "noise_floor_run": "FP64 with the CG SpMV summed over 16 lanes per row instead of 8",
        "wall_s": wall,
    }


def run_sloshing_adjoint(args):
    """Cost of the differentiation form on the 3-D sloshing tank with driven
    walls (tank 0.6 x 0.4 x 0.3 m, y vertical, water depth 0.2 m, l0 = 0.004
    unless --l0, walls driven along x with A = 0.01 m, f = 1.5 Hz): one
    rollout of `args.sloshing_adjoint` steps with a checkpoint every
    `args.every` steps, forward then backward, timed with CUDA events on the
    library's stream (no warm-up rollout: first-use allocations fall in the
    forward), the device memory in use after each, and the gradients with
    respect to the drive amplitude and frequency, the gravity scale, the
    viscosity and the initial velocities.  Loss: the time mean of the
    squared wall-probe pressure, the probe being the first wall layer's
    particles within 3 l0 of the point at height 0.1 m, mid-depth, on the
    +x wall (its mean pressure recorded after every step)."""
    import numpy as np
    import torch

    from mps_b200 import _lib
    from mps_b200 import workloads as W
    from mps_b200.adjoint import Rollout

    steps, every = int(args.sloshing_adjoint), int(args.every)
    l0 = args.l0 if args.l0 is not None else 0.004
    wl = W.sloshing3d(l0=l0, seed=1000, steps=steps)
    amp, freq, axis = wl.drive
    cfg = wl.config()
    prec = _lib.PREC_MIXED if args.precision == "mixed" else _lib.PREC_FP64
    domain = [cfg.domain_max[d] for d in range(3)]
    probe = probe_mask(wl.pos, wl.types, l0, domain, height=0.1, zc=0.5 * domain[2])
    roll = Rollout(cfg, 3, wl.pos, wl.types, steps, every=every, precision=prec, drive_axis=axis, probe=probe)
    stream = torch.cuda.ExternalStream(roll.sess.stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    x, u, t = roll.forward(wl.vel, 1.0, cfg.viscosity, amp, freq)
    ev[1].record(stream)
    torch.cuda.synchronize()
    free, total = torch.cuda.mem_get_info()
    used_fwd = total - free
    series = roll.series.copy()
    loss = float(np.mean(series ** 2))
    ev[2].record(stream)
    dx0, du0, dgs, dnu, dA, df = roll.backward(np.zeros_like(x), np.zeros_like(u), 2.0 * series / steps)
    ev[3].record(stream)
    torch.cuda.synchronize()
    free, total = torch.cuda.mem_get_info()
    used_bwd = total - free
    roll.close()
    fwd = ev[0].elapsed_time(ev[1]) / steps
    bwd = ev[2].elapsed_time(ev[3]) / steps
    grads = {"dL_dA": float(dA), "dL_df": float(df), "dL_dgravity_scale": float(dgs), "dL_dnu": float(dnu),
             "dL_du0_l2": float(np.linalg.norm(du0))}
    return {"metric": "adjoint/forward cost per step, 3-D sloshing with driven walls",
            "workload": wl.name, "particles": int(wl.n), "fluid": int(wl.n_fluid), "precision": args.precision,
            "rollout_steps": steps, "checkpoint_every": every, "dt": cfg.dt, "drive": {"A": amp, "f": freq, "axis": axis},
            "fwd_ms_per_step": fwd, "backward_ms_per_step": bwd, "adjoint_over_fwd": bwd / fwd,
            "device_memory_in_use_gb": {"after_forward": used_fwd / 1e9, "after_backward": used_bwd / 1e9},
            "loss": loss, "probe_particles": int(probe.sum()),
            "probe_pressure_first_last": [float(series[0]), float(series[-1])],
            "gradients": grads, "all_finite": bool(np.all(np.isfinite(list(grads.values())))),
            "note": "backward = segment recompute from each checkpoint + per-step recompute and reverse pass "
                    "incl. the adjoint PPE solve"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward cost measurement")
    ap.add_argument("--l0", type=float, default=None,
                    help="particle spacing override (smaller cases for profiling)")
    ap.add_argument("--error-growth", type=int, default=0, metavar="STEPS",
                    help="instead of the throughput line: the mixed form's error growth against FP64 over "
                         "STEPS steps (l0 = 0.01 unless --l0), with the FP64 reordering noise floor")
    ap.add_argument("--sloshing-adjoint", type=int, default=0, metavar="STEPS",
                    help="instead of the throughput line: adjoint/forward cost of a STEPS-step rollout of the "
                         "3-D sloshing tank with driven walls (l0 = 0.004 unless --l0)")
    ap.add_argument("--every", type=int, default=25, help="checkpoint interval of --sloshing-adjoint")
    args = ap.parse_args()
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        if rank != 0:
            return 0
        v, sec, meta = reference_cpu_steps(args.steps, args.warmup)
        line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": WORKLOADS[args.workload] + "; timed on the CPU sample below",
                           "precision": "fp64", "parallelism": "OpenMP, host cores"},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": meta["cores"], "kind": meta["kind"],
                                 "sample": meta["sample"]},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if args.sloshing_adjoint > 0:
        if rank == 0:
            print(json.dumps(run_sloshing_adjoint(args)))
        return 0

    if args.error_growth > 0:
        if rank == 0:
            print(json.dumps(run_error_growth(args)))
        return 0

    res = run_b200(args, rank, world, local_rank)
    if rank == 0 and res is not None:
        print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
