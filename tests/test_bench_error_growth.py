"""CPU checks of the helpers behind `bench.py --error-growth` (the mixed
form's long-run accuracy report): relative errors of states, the binned
pressure field and the wall probe, on synthetic states of the dam-break
geometry."""
import numpy as np

import bench
from mps_b200 import types as T
from mps_b200 import workloads as W


def _state(wl, seed=0):
    rng = np.random.default_rng(seed)
    st = np.zeros(wl.n, dtype=T.particle_dtype(3))
    st["pos"] = wl.pos
    st["vel"] = rng.normal(size=(wl.n, 3))
    st["type"] = wl.types
    st["pressure"] = rng.uniform(0.0, 5000.0, size=wl.n)
    st["on_surface"] = (rng.uniform(size=wl.n) < 0.1).astype(st["on_surface"].dtype)
    return st


def test_state_errors_identical_and_perturbed():
    wl = W.dambreak("c1", seed=1000, l0=0.02)
    a = _state(wl)
    e = bench.state_errors(a, a)
    assert e == {"p_rel": 0.0, "v_rel": 0.0, "x_rel": 0.0, "surface_flags_differing": 0, "types_differing": 0}
    b = a.copy()
    b["pressure"] *= 1.0 + 1e-6
    b["on_surface"][:3] = 1 - b["on_surface"][:3]
    b["type"][np.nonzero(wl.types == 0)[0][0]] = 2   # one fluid particle ghosted
    e = bench.state_errors(b, a)
    assert abs(e["p_rel"] - 1e-6) < 1e-12
    assert e["v_rel"] == 0.0 and e["x_rel"] == 0.0
    assert e["surface_flags_differing"] == 3
    assert e["types_differing"] == 1


def test_grid_pressure_and_probe_on_the_dam_break():
    l0 = 0.01
    wl = W.dambreak("c1", seed=1000, l0=l0)
    cfg = wl.config()
    domain = [cfg.domain_max[d] for d in range(3)]
    st = _state(wl, seed=1)
    ssum, cnt = bench.grid_pressure(st, l0, domain)
    fluid = st["type"] == 0
    assert int(cnt.sum()) == int(fluid.sum())
    assert abs(ssum.sum() - st["pressure"][fluid].sum()) <= 1e-9 * st["pressure"][fluid].sum()
    probe = bench.probe_mask(wl.pos, wl.types, l0, domain)
    n = int(probe.sum())
    assert 10 <= n <= 60          # a disc of radius 3 l0 on one lattice layer: ~28 particles
    assert np.all(wl.types[probe] == 1)
    assert np.all(wl.pos[probe, 0] > domain[0])
    ob = bench.observables(st, probe)
    assert ob["fluid"] == int(fluid.sum())
    assert abs(ob["front_x"] - wl.pos[fluid, 0].max()) == 0.0
    assert abs(ob["probe_p"] - st["pressure"][probe].mean()) <= 1e-9 * ob["probe_p"]
