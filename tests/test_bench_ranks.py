"""bench.py's multi-rank contract on CPU (gloo, world size 2): every rank
runs an independent replica, the job's time is the maximum over ranks, the
value is the fluid particle-steps of all replicas per second of that time,
and the reference arm runs on rank 0 only (other ranks exit 0 at once)."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_body(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank                       # rank 1 is the slow one
    job = bench.max_over_ranks(ms, dist, "cpu")
    out[rank] = (job, bench.whole_job_value(1000, world, 4, job / 1e3))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_value_gloo():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_body, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        job, value = res[r]
        assert job == 15.0
        assert value == pytest.approx(1000 * world * 4 / 0.015)


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
