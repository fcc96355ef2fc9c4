"""The reference's own main.c (3-D OpenMP and 2-D variants), compiled
unchanged against the reference's own headers, links against libmps3d.so /
libmps2d.so with no missing symbol, loads the B200 libraries and runs up to
its argument check (no GPU work: without a deck it prints its usage and
exits 1).  This is the link line a maintainer of the reference uses to swap
its src/*.c for this library.  Compiled into a temporary directory; skipped
where the reference sources are absent."""
import os
import subprocess

import pytest

from conftest import REF_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = REF_DIR or ""


@pytest.mark.parametrize("variant,dim", [("mps_fluid3D_parallel", 3), ("mps_fluid2D", 2)])
def test_reference_main_links_against_the_dropin(variant, dim, tmp_path):
    src = os.path.join(REF, variant, "src", "main.c")
    if not os.path.exists(src):
        pytest.skip("reference sources absent")
    lib = os.path.join(ROOT, "mps_b200")
    exe = str(tmp_path / f"mps_main{dim}d")
    r = subprocess.run(["gcc", "-O2", "-I", os.path.join(REF, variant, "include"), src, "-L", lib, f"-lmps{dim}d",
                        f"-Wl,-rpath-link,{lib}", f"-Wl,-rpath,{lib}", "-lm", "-o", exe],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    deps = subprocess.run(["ldd", exe], capture_output=True, text=True, timeout=60).stdout
    assert os.path.join(lib, f"libmps{dim}d.so") in deps and os.path.join(lib, "libmps_b200.so") in deps, deps
    assert "not found" not in deps, deps
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Usage:" in r.stderr, (r.returncode, r.stderr)


@pytest.mark.parametrize("variant,dim", [("mps_fluid3D_parallel", 3), ("mps_fluid2D", 2)])
def test_every_reference_prototype_is_exported(variant, dim):
    """Every function the reference's public headers declare is exported by
    the drop-in library of that dimension under the same name."""
    import glob
    import re
    inc = os.path.join(REF, variant, "include")
    if not os.path.isdir(inc):
        pytest.skip("reference sources absent")
    names = set()
    for h in glob.glob(os.path.join(inc, "*.h")):
        t = open(h).read()
        t = re.sub(r"/\*.*?\*/", "", t, flags=re.S)
        t = re.sub(r"//[^\n]*", "", t)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([a-z_][a-z0-9_]*)\s*\([^;{]*\)\s*;", t, flags=re.M):
            names.add(m.group(1))
    assert len(names) >= 30
    nm = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "mps_b200", f"libmps{dim}d.so")],
                        capture_output=True, text=True, timeout=60).stdout.split()
    exported = set(nm[2::3])
    assert not (names - exported), sorted(names - exported)
