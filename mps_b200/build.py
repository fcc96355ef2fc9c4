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
    "libmps_b200.so": ["engine.cu"],
}


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


def build_oracle() -> None:
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_cuda(force=force, verbose=verbose)
    build_oracle()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
