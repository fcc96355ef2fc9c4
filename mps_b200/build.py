"""Builds the sm_100a CUDA library in-tree (``mps_b200/libmps_b200.so``).

    python -m mps_b200.build

nvcc flags: ``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3
--fmad=false``.  ``--fmad=false`` is required: the FP64 parity kernels must
not contract a*b+c into FMAs, which the reference's x86 build never does.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-lineinfo", "-O3", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-Xcompiler", "-ffp-contract=off"]

TARGETS = {
    "libmps_b200.so": ["engine.cu", "noalloc.cu"],
}
CXX = os.environ.get("MPS_CXX", "g++")
CC = os.environ.get("MPS_CC", "gcc")
HOST_FLAGS = ["-O2", "-ffp-contract=off", "-fPIC", "-Wall"]


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(force: bool = False, verbose: bool = False) -> list:
    deps = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    built = []
    for name, srcs in TARGETS.items():
        out = os.path.join(HERE, name)
        if not force and not _stale(out, deps):
            continue
        cmd = [NVCC, *ARCH, *FLAGS, "-shared", "-o", out] + [os.path.join(CSRC, s) for s in srcs]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {name}:\n{r.stdout}\n{r.stderr}")
        built.append(out)
    return built


def build_host(force: bool = False, verbose: bool = False) -> list:
    """The drop-in libraries libmps3d.so / libmps2d.so and the mps_sim3d /
    mps_sim2d command-line drivers, linked against libmps_b200.so."""
    deps = [os.path.join(CSRC, "dropin.cpp"), os.path.join(CSRC, "mps_sim.c"), os.path.join(HERE, "libmps_b200.so")]
    deps += glob.glob(os.path.join(ROOT, "include", "*.h"))
    built = []
    for dim in (3, 2):
        lib = os.path.join(HERE, f"libmps{dim}d.so")
        exe = os.path.join(HERE, f"mps_sim{dim}d")
        jobs = [
            (lib, [CXX, *HOST_FLAGS, "-std=c++17", "-shared", f"-DMPS_DIM={dim}", "-o", lib,
                   os.path.join(CSRC, "dropin.cpp"), f"-L{HERE}", "-lmps_b200", "-Wl,-rpath,$ORIGIN"]),
            (exe, [CC, *HOST_FLAGS, f"-DMPS_DIM={dim}", "-o", exe, os.path.join(CSRC, "mps_sim.c"),
                   f"-L{HERE}", f"-lmps{dim}d", "-lmps_b200", "-Wl,-rpath,$ORIGIN"]),
        ]
        for out, cmd in jobs:
            if not force and not _stale(out, deps + ([lib] if out == exe else [])):
                continue
            if verbose:
                print(" ".join(cmd))
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"build failed for {out}:\n{r.stdout}\n{r.stderr}")
            built.append(out)
    return built


def build_oracle(force: bool = False) -> None:
    cmd = ["make", "-C", os.path.join(ROOT, "oracle")] + (["-B"] if force else [])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_cuda(force=force, verbose=verbose)
    build_host(force=force, verbose=verbose)
    build_oracle(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
