"""Throughput of the MPS time step on B200: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c2] [--precision both|mixed|fp64]

A step is one full MPS time step (simulation.c:19-118 of the reference) of
the 3-D dam break named by --workload, device-resident: explicit viscosity
and collision, the cell-sort neighbour search, number density and surface
flags, PPE assembly, IC(0) factorisation and the PCG solve to the absolute
tolerance 1e-9, the pressure gradient and the correction.  `value` is fluid
particle-steps/s over all ranks (each rank runs an independent replica with
its own seed: the time step has no partition that avoids a halo exchange
per operator and changes the IC(0) preconditioner).  The workload's PPE
matrix alone is 2.7 GB at c2, far above the 126 MB L2, so consecutive steps
do not run from cache.

By default every step (warm-up, timed, profiled, and every e2e call) starts
from the same state, the workload's initial state after the first
neighbour search: one pass of the hot path over one batch of input.  The c2
dam break from its jittered lattice goes unstable after about 15 steps of
the reference's scheme (particles at hundreds of m/s near the side walls,
then a NaN in the PPE), so a rollout long enough for the timing window
would time broken flow.  The device-side checkpoint load is inside the
timed region; the e2e arm restores its host arrays between the timed calls.
--rollout times consecutive steps instead.

Other keys: `roofline` for the dominant kernel (the IC(0) colour sweep
k_sweep_colour, with the CG SpMV beside it; CUDA events on the library's
stream in two profiled steps after the timed ones), `cpu_baseline` (the
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
    "c2": "3-D dam break, tank 1.6x0.6x0.6 m, column 0.4x0.6x0.3 m, l0=0.0035 m, 2,854,670 particles "
          "(1,656,990 fluid), dt 3.5e-4, ICCG tol 1e-9",
}
# The mixed form's stopping rule, as the engine applies it (engine.cu, mixed_solve).
MIXED_STOP = ("||b - A x|| <= 4 u || |b| + |A| |x| || (u = 2^-53: four times the rounding floor of an FP64 "
              "residual, where the FP64 form's solve ends), or two reliable updates in a row that do not halve it")
# Steps of the reference's CPU build timed by --impl reference: one step of
# the c2 dam break takes about two minutes on 16 host cores, so the
# reference arm times a bounded window of the first REF_WINDOW steps.
REF_WINDOW = 3


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

def reference_cpu_steps(workload: str, steps: int, warmup: int, l0=None, seed: int = 1000, restart: bool = True):
    """Times `steps` reference simulation_step calls (after `warmup` untimed
    ones) on the workload (the same seeded initial state as the GPU arm's
    rank 0); with `restart`, every call starts from the initial particles
    and list, restored between the timed calls, as the GPU arm's steps do.
    Returns (fluid particle-steps/s, seconds/step, meta)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(host_cores()))
    from mps_b200 import config as CF
    from mps_b200 import types as T
    from mps_b200 import workloads as W
    from oracle.pyoracle import Oracle, Reference

    wl = W.dambreak(workload, l0=l0, seed=seed)
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
    if restart:
        arr0, cnt0, nb0 = hp.arr.copy(), nl.count.copy(), nl.neighbors.copy()

    def restore():
        if restart:
            hp.arr[:] = arr0
            nl.count[:] = cnt0
            nl.neighbors[:] = nb0

    for s in range(warmup):
        restore()
        ref.step(hp, nl, cl, s + 1)
    dt = 0.0
    for s in range(steps):
        restore()
        t0 = time.perf_counter()
        ref.step(hp, nl, cl, warmup + s + 1)
        dt += time.perf_counter() - t0
    ref.lib.cell_list_free(cl)
    meta = {"kind": kind, "cores": int(os.environ["OMP_NUM_THREADS"]),
            "sample": f"{wl.name} ({wl.n} particles, {wl.n_fluid} fluid), {steps} reference "
                      f"simulation_step call(s) after {warmup} warm-up, "
                      + ("each from the initial state (restored between calls, not timed), " if restart else
                         "consecutive from the initial state, ") +
                      "OpenMP build of mps_fluid3D_parallel compiled from source; n0/lambda from the oracle's "
                      "cell-list form of particle_system_calc_initial_params (bit-identical, not timed)"}
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
                "reasons": sorted(reasons), "samples": len(sm), "sm_samples": sm}


def merge_clocks(parts):
    """One clocks record over several sampled timed regions."""
    parts = [p for p in parts if p]
    if not parts:
        return None
    sm = [v for p in parts for v in p.get("sm_samples", [])]
    mx = next((p["sm_max_mhz"] for p in parts if p.get("sm_max_mhz")), None)
    reasons = sorted({r for p in parts for r in p.get("reasons", [])})
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
            "samples": len(sm), "regions": len(parts)}


# ---------------------------------------------------------------------------
# roofline of the dominant kernel
# ---------------------------------------------------------------------------

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0}, "fallback"


def ncu_traffic(kernel: str, form: str):
    """(DRAM bytes, algorithmic bytes) of `kernel` in precision form `form`
    from a committed ncu summary (profiles/*.md lines
    'traffic_per_launch_bytes <kernel> <form> <dram bytes> <algorithmic bytes>');
    None when absent.  The bench scales the ratio to its own workload."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for name in sorted(os.listdir(d)):
        if not name.endswith(".md"):
            continue
        for line in open(os.path.join(d, name)):
            t = line.strip().strip("`").split()
            if len(t) == 5 and t[0] == "traffic_per_launch_bytes" and t[1] == kernel and t[2] == form:
                return float(t[3]), float(t[4])
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


def time_form(wl, cfg, prec, args, torch, dist, barrier, lib):
    """Times one precision form on the workload: a session from the initial
    state, args.warmup untimed steps (the first one's pressures kept for the
    mixed-vs-FP64 check), then args.steps steps timed with CUDA events on
    the library's stream (max over ranks), then min(steps, 2) profiled steps
    (CUDA events around every CG-loop kernel group; not part of the timed
    figure).  Returns a dict of the form's figures."""
    import numpy as np

    from mps_b200 import types as T
    from mps_b200.session import Session

    hp = T.HostParticles(3, wl.pos, wl.vel, wl.types)
    sess = Session(cfg, 3, hp.n, precision=prec, refine_tolerance=args.refine_tolerance)
    sess.upload(hp)
    n0, lam, _ = sess.compute_initial_params()
    sess.neighbor_search()
    # restart mode: every step starts from this checkpoint of the initial
    # state (its neighbour structure included), kept in device memory; the
    # load is a device-to-device copy inside the timed region
    ckpt = None
    if args.restart:
        ckpt = torch.empty(sess.state_bytes(), dtype=torch.uint8, device="cuda")
        sess.state_save(ckpt.data_ptr())

    def one_step():
        if ckpt is not None:
            sess.state_load(ckpt.data_ptr())
        sess.step(1)

    one_step()
    p1 = sess.pressure()
    for _ in range(args.warmup - 1):
        one_step()
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(sess.stream)
    sess.reset_metrics()
    per_step = []
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device()) if args.rank == 0 else None
    l0 = lib.mps_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        one_step()
        m = sess.metrics()   # host-side copy; each step already ends in a host sync
        per_step.append((m["ppe_iterations"], m["ppe_true_residual"], m["ppe_bnorm"], m["ppe_rounding_floor"],
                         m["ppe_outer"]))
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = lib.mps_launch_count() - l0
    ms = e0.elapsed_time(e1)
    clk = clocks.stop() if clocks else None
    met = sess.metrics()
    sess.reset_metrics()
    sess.set_profiling(True)
    for _ in range(min(args.steps, 2)):
        one_step()
    torch.cuda.synchronize()
    pmet = sess.metrics()
    sess.set_profiling(False)
    # a short rollout window from the initial state: steps 2..6 timed, the
    # flow past its start-up transient and before the late instability
    window = None
    if ckpt is not None and args.window > 0:
        sess.state_load(ckpt.data_ptr())
        sess.step(1)
        torch.cuda.synchronize()
        w0 = torch.cuda.Event(enable_timing=True)
        w1 = torch.cuda.Event(enable_timing=True)
        its = []
        w0.record(stream)
        for _ in range(args.window):
            sess.step(1)
            its.append(sess.metrics()["ppe_iterations"])
        w1.record(stream)
        torch.cuda.synchronize()
        window = {"steps": f"2..{1 + args.window} of one rollout", "ms_per_step": w0.elapsed_time(w1) / args.window,
                  "ppe_iterations_per_step": float(np.mean(its))}
    sess.close()
    ms_max = max_over_ranks(ms, dist, "cuda")
    it = np.array([r[0] for r in per_step], dtype=np.float64)
    tr = np.array([r[1] for r in per_step])
    bn = np.array([r[2] for r in per_step])
    fl = np.array([r[3] for r in per_step])
    return {"ms": ms_max, "ms_per_step": ms_max / args.steps, "window": window, "launches": int(launches), "clocks": clk,
            "n0": n0, "lambda": lam, "p_step1": p1, "met": met, "pmet": pmet,
            "iterations_per_step": float(it.mean()), "iterations_total": int(it.sum()),
            "outer_updates_per_step": float(np.mean([r[4] for r in per_step])),
            "true_residual": {"mean": float(tr.mean()), "max": float(tr.max()),
                              "relative_mean": float(np.mean(tr / bn)), "relative_max": float(np.max(tr / bn)),
                              "over_rounding_floor_mean": float(np.mean(tr / fl))}}


def sweep_bytes(pmet, fp32: bool) -> dict:
    """Algorithmic bytes of one forward and one backward IC(0) sweep (all 8
    colour launches of k_sweep_colour): every cross-cell factor entry once
    (value + int32 column), every in-cell block-inverse entry once, and per
    row the run bounds (2 x 4 B), rhs read, the partial sum written and read
    back, and the result written (4 x 8 B); the gathers of the solution
    vector are served on chip."""
    vb = 4.0 if fp32 else 8.0
    e = float(pmet["n_eq"])
    inv = float(pmet["sweep_inverse_entries"])
    fwd = (vb + 4.0) * pmet["sweep_cross_lo"] + vb * inv + 40.0 * e
    bwd = (vb + 4.0) * pmet["sweep_cross_up"] + vb * inv + 40.0 * e
    return {"forward": fwd, "backward": bwd}


def pcg_iter_bytes(pmet, fp32: bool, diff: bool) -> float:
    """Algorithmic bytes of one iteration of the persistent ICCG kernel
    (k_pcg): the SpMV (matrix value + int32 column per nonzero, row
    pointers, p and z read, Ap and the new p written, the row sums of the
    difference form), the forward sweep (lower cross entries, the block
    inverses, r and x read and written, p and Ap read, y written), the
    backward sweep (upper cross entries, the block inverses, y and r read, z
    written) and the per-cell structure of both sweeps (jagged-diagonal
    starts and row ranks, about 6 B per row); the gathers of p, y and z are
    served on chip."""
    vb = 4.0 if fp32 else 8.0
    e = float(pmet["n_eq"])
    z = float(pmet["nnz"])
    inv = float(pmet["sweep_inverse_entries"])
    spmv = (vb + 4.0) * z + 4.0 * e + 32.0 * e + (8.0 * e if diff else 0.0)
    fwd = (vb + 4.0) * pmet["sweep_cross_lo"] + vb * inv + 56.0 * e
    bwd = (vb + 4.0) * pmet["sweep_cross_up"] + vb * inv + 24.0 * e
    return spmv + fwd + bwd + 12.0 * e


def run_b200(args, rank: int, world: int, local_rank: int):
    import numpy as np
    import torch

    from mps_b200 import _lib
    from mps_b200 import workloads as W

    torch.cuda.set_device(local_rank)
    args.rank = rank
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()

    wl = W.dambreak(args.workload, seed=1000 + rank, l0=args.l0)
    cfg = wl.config()
    lib = _lib.load()
    forms = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    res = {}
    for f in forms:
        prec = _lib.PREC_MIXED if f == "mixed" else _lib.PREC_FP64
        res[f] = time_form(wl, cfg, prec, args, torch, dist, barrier, lib)
    head = forms[0]
    hr = res[head]
    value = whole_job_value(wl.n_fluid, world, args.steps, hr["ms"] / 1e3)

    e2e = None if args.no_e2e else run_e2e(wl, cfg, args, torch, dist, head)
    adjoint = None
    if world == 1 and not args.no_adjoint:
        adjoint = run_adjoint_cost(wl, cfg, _lib.PREC_MIXED if head == "mixed" else _lib.PREC_FP64, torch)

    result = None
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        peak = float(peaks.get("hbm_gbs", 6650.0))
        kern = {}
        roof = []
        for f in forms:
            pm = res[f]["pmet"]
            fp32 = f == "mixed"
            if pm.get("prof_pcg_launches", 0) > 0:
                # persistent ICCG kernel: one launch per batch of iterations
                ipl = pm["prof_pcg_iterations"] / pm["prof_pcg_launches"]
                ms_launch = pm["prof_pcg_ms"] / pm["prof_pcg_launches"]
                ms_iter = pm["prof_pcg_ms"] / max(pm["prof_pcg_iterations"], 1)
                b_iter = pcg_iter_bytes(pm, fp32, fp32)
                kern[f] = {"k_pcg_ms_per_iteration": ms_iter, "k_pcg_iterations_per_launch": ipl,
                           "spmv_phase_ms": pm["prof_spmv_ms"] / max(pm["prof_spmv_launches"], 1),
                           "forward_phases_ms": pm["prof_fwd_ms"] / max(pm["prof_fwd_sweeps"], 1),
                           "backward_phases_ms": pm["prof_bwd_ms"] / max(pm["prof_bwd_sweeps"], 1)}
                t = ncu_traffic("k_pcg", f)
                ach = b_iter / (ms_iter / 1e3) / 1e9
                roof.append({"form": f, "kernel": "k_pcg", "bound": "hbm", "achieved": ach, "peak": peak,
                             "unit": "GB/s", "frac": ach / peak,
                             "traffic": None if t is None else t[0] / t[1] * b_iter * ipl,
                             "algorithmic_bytes_per_iteration": b_iter,
                             "algorithmic_bytes_per_launch": b_iter * ipl, "iterations_per_launch": ipl,
                             "ms_per_launch": ms_launch, "ms_per_iteration": ms_iter})
                continue
            nnz_mean = pm["prof_nnz_sum"] / max(pm["prof_iterations"], 1)
            rows_mean = pm["prof_rows_sum"] / max(pm["prof_iterations"], 1)
            spmv_ms = pm["prof_spmv_ms"] / max(pm["prof_spmv_launches"], 1)
            fwd_ms = pm["prof_fwd_ms"] / max(pm["prof_fwd_sweeps"], 1)
            bwd_ms = pm["prof_bwd_ms"] / max(pm["prof_bwd_sweeps"], 1)
            vec_ms = pm["prof_vec_ms"] / max(pm["prof_iterations"], 1)
            # SpMV: matrix value + column per nonzero, row pointer, p and Ap per row (FP64),
            # and in the mixed form's difference form the FP64 row sum
            spmv_b = ((4.0 if fp32 else 8.0) + 4.0) * nnz_mean + (28.0 if fp32 else 20.0) * rows_mean
            sb = sweep_bytes(pm, fp32)
            sw_b = 0.5 * (sb["forward"] + sb["backward"])
            sw_ms = 0.5 * (fwd_ms + bwd_ms)
            kern[f] = {"k_cg_spmv_ms": spmv_ms, "ic0_forward_sweep_ms(8 colour launches)": fwd_ms,
                       "ic0_backward_sweep_ms(8 colour launches)": bwd_ms, "cg_axpy_ms": vec_ms}
            tsw = ncu_traffic("k_sweep_colour", f)
            tsp = ncu_traffic("k_cg_spmv", f)
            if sw_ms > 0:
                roof.append({"form": f, "kernel": "k_sweep_colour", "bound": "hbm",
                             "achieved": sw_b / (sw_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": sw_b / (sw_ms / 1e3) / 1e9 / peak,
                             "traffic": None if tsw is None else tsw[0] / tsw[1] * sw_b,
                             "algorithmic_bytes_per_launch": sw_b / 8.0, "launches_per_sweep": 8,
                             "algorithmic_bytes_per_sweep": sw_b, "ms_per_sweep": sw_ms})
            if spmv_ms > 0:
                roof.append({"form": f, "kernel": "k_cg_spmv", "bound": "hbm",
                             "achieved": spmv_b / (spmv_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": spmv_b / (spmv_ms / 1e3) / 1e9 / peak,
                             "traffic": None if tsp is None else tsp[0] / tsp[1] * spmv_b,
                             "algorithmic_bytes_per_launch": spmv_b, "ms_per_launch": spmv_ms})
        top = dict(roof[0])
        top.update({"peak_source": f"{peak_kind} hbm_gbs",
                    "timing": "CUDA events on the library stream around every launch of the ICCG loop's kernels "
                              "(k_pcg: one launch per batch of iterations; the launch-per-colour form: every colour "
                              "sweep and SpMV), over min(steps, 2) profiled steps right after the timed region",
                    "others": roof[1:]})
        cpu = None
        if world == 1 and not args.no_cpu:
            v, sec, meta = reference_cpu_steps(args.workload, args.cpu_steps, 0, l0=args.l0, restart=args.restart)
            cpu = {"value": v, "unit": UNIT, "cores": meta["cores"], "kind": meta["kind"], "sample": meta["sample"],
                   "seconds_per_step": sec}
        forms_out = {}
        for f in forms:
            r = res[f]
            forms_out[f] = {"ms_per_step": r["ms_per_step"],
                            "fluid_particle_steps_per_s": whole_job_value(wl.n_fluid, world, args.steps,
                                                                          r["ms"] / 1e3),
                            "ppe_iterations_per_step": r["iterations_per_step"],
                            "ppe_iterations_per_s": r["iterations_total"] / (r["ms"] / 1e3),
                            "reliable_updates_per_step": r["outer_updates_per_step"],
                            "true_residual": r["true_residual"],
                            "stage_ms_last_step": {"ops": r["met"]["ms_ops"], "assembly": r["met"]["ms_assembly"],
                                                   "factor": r["met"]["ms_factor"], "solve": r["met"]["ms_solve"]},
                            "kernel_ms": kern[f], "gpu_launches": r["launches"], "clocks": r["clocks"],
                            "rollout_window": r["window"]}
        extra = {}
        if len(forms) == 2:
            pm, pf = res["mixed"]["p_step1"], res["fp64"]["p_step1"]
            wm, wf = res["mixed"]["window"], res["fp64"]["window"]
            extra = {"mixed_over_fp64_speedup": res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"],
                     "mixed_over_fp64_speedup_rollout_window": (wf["ms_per_step"] / wm["ms_per_step"])
                     if wm and wf else None,
                     "step1_pressure_rel_l2_mixed_vs_fp64": float(np.linalg.norm(pm - pf) / np.linalg.norm(pf)),
                     "equal_residual": "both forms' true residual ||b - A x|| per step is in forms.*.true_residual; "
                                       "FP64 stops on the reference's recursive test (sqrt(r.r) < 1e-9), the mixed "
                                       "form on its true residual (" + MIXED_STOP + ")"}
        clk_all = [res[f]["clocks"] for f in forms if res[f]["clocks"]]
        result = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": hr["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 storage + f64" if head == "mixed" else "f64",
            "data": "synthetic",
            "config": {
                "workload": WORKLOADS.get(args.workload, args.workload) if args.l0 is None
                else f"{args.workload} geometry at l0={args.l0}",
                "particles_per_gpu": wl.n,
                "fluid_per_gpu": wl.n_fluid,
                "precision": head,
                "forms_timed": forms,
                "parallelism": f"replicas x{world}",
                "steps_from": "every step restarts from the initial state after the first neighbour search"
                              if args.restart else "consecutive steps of one rollout",
                "l2": "inputs larger than L2 (PPE matrix ~%.1f GB per replica)"
                      % ((12.0 * hr["met"]["nnz"]) / 1e9),
                "n0": hr["n0"],
                "lambda": hr["lambda"],
            },
            "total_particle_steps_per_s": wl.n * world * args.steps / (hr["ms"] / 1e3),
            "ppe_iterations_per_step": hr["iterations_per_step"],
            "ppe_iterations_per_s": hr["iterations_total"] / (hr["ms"] / 1e3),
            "forms": forms_out,
            **extra,
            "roofline": top,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "adjoint": adjoint,
            "gpu_launches": int(hr["launches"]),
            "clocks": merge_clocks(clk_all),
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


def run_e2e(wl, cfg, args, torch, dist, form):
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
    prec = _lib.PREC_MIXED if form == "mixed" else _lib.PREC_FP64
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
    # restart mode: every call starts from the initial particles and list,
    # restored on the host between the timed calls
    nbv = nb_buf.numpy().reshape(n, m)
    mc0 = int(cnt.max())
    if args.restart:
        parts0, cnt0, nb0 = parts.copy(), cnt.copy(), nbv[:, :mc0].copy()

    def restore():
        if args.restart:
            parts[:] = parts0
            cnt[:] = cnt0
            nbv[:, :mc0] = nb0

    lib.simulation_step(C.byref(ps), C.byref(nl), cl, 1)           # warm-up call
    steps = args.steps
    h2d = d2h = 0
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    # the drop-in calls are synchronous (host copies in and out), so CUDA
    # events on the idle current stream, after a device synchronize, bracket
    # exactly each call; the restores between calls are not timed
    wall = 0.0
    for k in range(steps):
        restore()
        mc_in = int(cnt.max())
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        lib.simulation_step(C.byref(ps), C.byref(nl), cl, 2 + k)
        ev1.record()
        torch.cuda.synchronize()
        wall += ev0.elapsed_time(ev1) / 1e3
        mc_out = int(cnt.max())
        # bytes copied by the call: AoS particles and the counts both ways,
        # the used columns of the list (pitched copy), the cell chains back
        h2d += n * dt_p.itemsize + 4 * n + 4 * n * mc_in
        d2h += n * dt_p.itemsize + 4 * n + 4 * n * mc_out + 4 * cl.contents.total_cells + 4 * n
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
            "precision": form}


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
    prec = _lib.PREC_FP64 if args.precision == "fp64" else _lib.PREC_MIXED
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
            "workload": wl.name, "particles": int(wl.n), "fluid": int(wl.n_fluid),
            "precision": "fp64" if args.precision == "fp64" else "mixed",
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
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: the mixed form (value) and the FP64 form timed on the same workload")
    ap.add_argument("--refine-tolerance", type=float, default=0.0,
                    help="mixed form: also stop at ||b - A x|| <= this * ||b|| (0: off)")
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--window", type=int, default=5,
                    help="restart mode: also time this many consecutive steps (2..window+1) of one rollout per form")
    ap.add_argument("--rollout", dest="restart", action="store_false",
                    help="time consecutive steps of one rollout instead of restarting every step from the initial "
                         "state (the c2 dam break from its lattice state goes unstable after about 15 steps)")
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
        nsteps = min(args.steps, REF_WINDOW)
        v, sec, meta = reference_cpu_steps(args.workload, nsteps, 0, l0=args.l0, restart=args.restart)
        meta["sample"] += (f"; a bounded window of {nsteps} step(s) instead of {args.steps} after {args.warmup} "
                           "warm-up (no warm-up: the reference allocates its PPE buffers in every call)")
        line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "same_config": True, "timed_steps": nsteps,
                "config": {"workload": WORKLOADS[args.workload] if args.l0 is None
                           else f"{args.workload} geometry at l0={args.l0}",
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
