"""Failure paths of the drop-in's host side, on the CPU (no GPU is touched).

  * capacity overflow: particle_system_add on a full system returns -1 and
    leaves the system as it was, as the reference's does (particle.c:40-43);
    checked call for call against the reference build (oracle/_ref);
  * a corrupt or missing particles.txt: the mps_sim3d / mps_sim2d command
    line stops with exit status 1 and the reference's message before any
    device work (main.c:20-85: a missing file, a count line that is not a
    positive integer).
"""
import ctypes as C
import os
import subprocess

import pytest

from mps_b200 import types as T
from mps_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("dim", [3, 2])
def test_capacity_overflow_matches_reference(dim):
    ref_path = os.path.join(ROOT, "oracle", "_ref", f"libref{dim}d.so")
    if not os.path.exists(ref_path):
        pytest.skip("the reference build (oracle/_ref) is absent")
    mine = C.CDLL(os.path.join(ROOT, "mps_b200", f"libmps{dim}d.so"))
    ref = C.CDLL(ref_path)
    PS = C.POINTER(T.ParticleSystem)
    DA = C.c_double * dim
    results = []
    for lib in (mine, ref):
        lib.particle_system_create.restype = PS
        lib.particle_system_create.argtypes = [C.c_int]
        lib.particle_system_add.restype = C.c_int
        lib.particle_system_add.argtypes = [PS, DA, DA, C.c_int]
        lib.particle_system_free.argtypes = [PS]
        ps = lib.particle_system_create(2)
        rc = [lib.particle_system_add(ps, DA(*[0.1 * (k + 1)] * dim), DA(*[0.0] * dim), 0) for k in range(4)]
        results.append((rc, ps.contents.num, ps.contents.capacity))
        lib.particle_system_free(ps)
    assert results[0] == results[1]
    assert results[0] == ([0, 1, -1, -1], 2, 2)


def _deck(tmp_path, dim):
    wl = W.small_dambreak3d(l0=0.04, seed=2) if dim == 3 else W.small_dambreak2d(l0=0.04, seed=2)
    cal = wl.write(str(tmp_path))
    return cal, os.path.join(str(tmp_path), "particles.txt")


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("content,message", [
    (None, "cannot open particle file"),
    ("# only a comment\n", "invalid particle count"),
    ("abc\nxyz 1\n", "invalid particle count"),
    ("0\n", "invalid particle count"),
    ("-5\n", "invalid particle count"),
])
def test_corrupt_particle_file_stops_cli(dim, content, message, tmp_path):
    exe = os.path.join(ROOT, "mps_b200", f"mps_sim{dim}d")
    if not os.path.exists(exe):
        pytest.skip("the command line driver is not built")
    cal, parts = _deck(tmp_path, dim)
    assert os.path.exists(parts)
    if content is None:
        os.remove(parts)
    else:
        with open(parts, "w") as f:
            f.write(content)
    r = subprocess.run([exe, cal], capture_output=True, text=True, timeout=60, cwd=str(tmp_path))
    assert r.returncode == 1, (r.stdout, r.stderr)
    assert message in r.stderr
