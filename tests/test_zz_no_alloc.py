"""mps_cell_sort_noalloc, the cell sort for callers that cannot allocate
device memory (see include/mps_b200.h), against the session's neighbour
search: same cell index for every particle, same particles in every cell in
the same order (the reference's chain order), two calls in a row on
different inputs through the same static scratch array.

Kept in its own file, named to be collected last, so that a run stopping
at the first failure has already run every other test.  It passes alone in
a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from mps_b200 import config as CF
from mps_b200 import types as T
from mps_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _grid(cfg, dim):
    """cell_list_create's grid (neighbor_search.c:92-122) for the list radius."""
    from mps_b200 import _lib
    re = CF.neighbor_radius(cfg)
    g = _lib.MpsGrid()
    g.dim = dim
    g.cell_size = re
    margin = 4.0 * re
    for d in range(dim):
        g.origin[d] = cfg.domain_min[d] - margin
        span = (cfg.domain_max[d] + margin) - g.origin[d]
        g.dims[d] = int(span / re) + 2
    return g


def _expected(cfg, dim, wl):
    """Cell index and per-cell chains from the existing session entry points."""
    from mps_b200.session import Session
    hp = T.HostParticles(dim, wl.pos, wl.vel, wl.types)
    with Session(cfg, dim, hp.n) as s:
        s.upload(hp)
        s.set_initial_params(1.0, 1.0, 0)
        s.neighbor_search()
        cell = s.cell_index()
        g = _grid(cfg, dim)
        total = int(np.prod([g.dims[d] for d in range(dim)]))
        head, nxt = s.cell_links(total)
    return cell, head, nxt, total


def _call(lib, g, wl, dim, torch):
    n = wl.n
    pos = torch.tensor(np.ascontiguousarray(wl.pos, dtype=np.float64).ravel(), device="cuda")
    typ = torch.tensor(np.ascontiguousarray(wl.types, dtype=np.int32), device="cuda")
    total = int(np.prod([g.dims[d] for d in range(dim)]))
    cell = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    order = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    start = torch.full((total + 1,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.mps_cell_sort_noalloc(C.byref(g), pos.data_ptr(), typ.data_ptr(), n, cell.data_ptr(),
                                   order.data_ptr(), start.data_ptr(), stream)
    torch.cuda.synchronize()
    return rc, cell.cpu().numpy(), order.cpu().numpy(), start.cpu().numpy()


def _check(cell, order, start, exp_cell, head, nxt, total, n):
    assert np.array_equal(cell, exp_cell)
    nbinned = int((exp_cell >= 0).sum())
    assert start[total] == nbinned
    for c in np.nonzero(head >= 0)[0]:
        chain = []
        j = head[c]
        while j >= 0:
            chain.append(j)
            j = nxt[j]
        assert np.array_equal(order[start[c]:start[c + 1]], np.array(chain, dtype=np.int32)), c
    assert np.array_equal(order[nbinned:], np.nonzero(exp_cell < 0)[0].astype(np.int32))
    assert np.array_equal(np.sort(order), np.arange(n, dtype=np.int32))


def test_cell_sort_noalloc_matches_session_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mps_b200 import _lib
    lib = _lib.load()
    runs = [W.small_dambreak3d(l0=0.02, seed=31), W.small_dambreak3d(l0=0.02, seed=32)]
    # a ghost, to exercise the unbinned tail
    runs[1].types[5] = T.GHOST
    for wl in runs:
        cfg = wl.config()
        exp_cell, head, nxt, total = _expected(cfg, 3, wl)
        g = _grid(cfg, 3)
        rc, cell, order, start = _call(lib, g, wl, 3, torch)
        assert rc == 0
        _check(cell, order, start, exp_cell, head, nxt, total, wl.n)


def test_cell_sort_noalloc_matches_session_twice_2d():
    """The 2-D grid (cell = iy * nx + ix, positions two per particle)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mps_b200 import _lib
    lib = _lib.load()
    runs = [W.small_dambreak2d(l0=0.01, seed=33), W.small_dambreak2d(l0=0.01, seed=34)]
    runs[0].types[7] = T.GHOST
    for wl in runs:
        cfg = wl.config()
        exp_cell, head, nxt, total = _expected(cfg, 2, wl)
        g = _grid(cfg, 2)
        rc, cell, order, start = _call(lib, g, wl, 2, torch)
        assert rc == 0
        _check(cell, order, start, exp_cell, head, nxt, total, wl.n)


def test_cell_sort_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mps_b200 import _lib
    lib = _lib.load()
    g = _lib.MpsGrid()
    g.dim = 3
    g.cell_size = 1.0
    g.dims[0], g.dims[1], g.dims[2] = 100, 100, 100     # 1e6 cells > the static limit
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = lib.mps_cell_sort_noalloc(C.byref(g), buf.data_ptr(), buf.data_ptr(), 1, buf.data_ptr(),
                                   buf.data_ptr(), buf.data_ptr(), 0)
    assert rc == -1
