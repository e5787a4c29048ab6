"""The N > 1 path of bench.py on CPU: replicas only (every rank computes its
own copy of the workload; no data-path collective), so what the ranks share
is the timing -- the job takes as long as its slowest rank -- and the
reference arm, which rank 0 alone runs.  Two gloo ranks on 127.0.0.1."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks_of(values[rank], dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        values = [12.5, 40.25]
        mp.start_processes(_rank_main, args=(2, _free_port(), values, out), nprocs=2, join=True,
                           start_method="spawn")
        assert dict(out) == {0: 40.25, 1: 40.25}


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks_of(3.0, None, "cpu") == 3.0


def test_replica_rate_counts_every_rank():
    import bench
    # 4 replicas x 3 energies x 2 steps in 500 ms (the slowest rank)
    assert bench.replica_rate(4, 3, 2, 500.0) == pytest.approx(48.0)


def test_reference_arm_runs_on_rank_0_only(capsys):
    import argparse

    import bench
    args = argparse.Namespace(steps=1, warmup=0, gpus=2)
    assert bench.run_reference(args, 1, 2) == 0
    assert capsys.readouterr().out == ""


def test_reference_arm_declines_boxes(capsys):
    import argparse
    import json

    import bench
    old = bench.WORKLOAD
    bench.WORKLOAD = "boxes"
    try:
        assert bench.run_reference(argparse.Namespace(steps=1, warmup=0, gpus=1), 0, 1) == 0
    finally:
        bench.WORKLOAD = old
    line = json.loads(capsys.readouterr().out)
    assert line["impl"] == "reference" and "unavailable" in line
