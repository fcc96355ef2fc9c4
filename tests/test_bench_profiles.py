"""The ncu traffic figures bench.py reads from the committed profile
summaries: every kernel and precision form that the bench line's roofline
reports has a 'traffic_per_launch_bytes' line, and each gives DRAM bytes
within a plausible multiple of its algorithmic bytes (a figure below the
algorithmic bytes, or far above them, would be a transcription error)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.mark.parametrize("kernel", ["k_sweep_colour", "k_cg_spmv"])
@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_traffic_line_for_every_roofline_entry(kernel, form):
    import bench

    t = bench.ncu_traffic(kernel, form)
    assert t is not None, (kernel, form)
    dram, algo = t
    assert algo > 0
    assert 0.95 <= dram / algo <= 3.0, (kernel, form, dram / algo)


def test_missing_entry_is_none():
    import bench

    assert bench.ncu_traffic("k_no_such_kernel", "fp64") is None
