"""Host logic of `bench.py --gpus N` (one process per GPU, N independent
replicas): the timed value of every rank is the maximum over the ranks, and
the reference arm runs on rank 0 only.  Two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        out[rank] = bench.max_over_ranks(torch, 1.5 + rank)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_timed_value_is_the_max_over_ranks():
    world = 2
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_without_a_group_the_value_is_unchanged():
    import bench
    assert bench.max_over_ranks(torch, 3.25) == 3.25


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(nx=8, ny=8, nz=8, steps=1, warmup=0, gpus=2)
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
