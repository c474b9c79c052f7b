"""The multi-rank path of bench.py (independent replicas, one reduction of
the step time) on two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        val = bench.whole_job_tflops(3e12, world, ms)
        out[rank] = (ms, val)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1]
    ms, val = out[0]
    assert ms == 2.5
    assert abs(val - 3e12 * 2 / 2.5e-3 / 1e12) < 1e-9


def test_single_rank_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert abs(bench.whole_job_tflops(1e12, 1, 1.0) - 1000.0) < 1e-9  # 1 TFLOP in 1 ms


def test_reference_arm_runs_on_rank0_only(capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    class A:
        steps, warmup = 1, 0
    assert bench.run_reference(A(), 1, 2) is None
    assert capsys.readouterr().out == ""
