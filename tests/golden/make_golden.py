"""Generate the committed golden fixtures from the reference's shipped outputs.

Reads the 3-D dam-break trajectory that the reference ships
(mps_fluid3D_parallel/output/output_000{000,100,200}.csv, produced by its
examples/dambreak deck) and stores every row's eight columns as float64
arrays in dambreak3d_golden.npz.  Run in a container that has the reference
checked out; the GPU hosts only read the .npz.

    python tests/golden/make_golden.py REF_DIR     (or MPS_REFERENCE_DIR=... python ...)
"""
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MPS_REFERENCE_DIR", "")
HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if not REF or not os.path.isdir(REF):
        sys.exit("usage: make_golden.py REF_DIR (the reference checkout; or set MPS_REFERENCE_DIR)")
    out = {}
    for step in (0, 100, 200):
        path = os.path.join(REF, "mps_fluid3D_parallel", "output", f"output_{step:06d}.csv")
        a = np.loadtxt(path, delimiter=",", skiprows=1)
        out[f"step{step}"] = a
    np.savez_compressed(os.path.join(HERE, "dambreak3d_golden.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
