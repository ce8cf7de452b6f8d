"""The multi-GPU path of bench.py runs one independent replica per rank ("replicas only": the
iteration's only cross-walker coupling, the MinSR Gram, is solved per GPU). Its one collective is
the max over ranks of the step time; the whole-job value is N replicas / that time. Checked here
with world_size-2 gloo process groups on the CPU, and the reference arm's rank > 0 exit."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 3.0 * rank)  # rank 1 is the slower replica
        e2e = bench.max_over_ranks(20.0 - rank)       # rank 0 is the slower one here
        out[rank] = (ms, e2e, bench.job_throughput(ms, world))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        ms, e2e, v = out[r]
        assert ms == 13.0 and e2e == 20.0
        assert v == pytest.approx(2 * 1000.0 / 13.0)


def test_max_over_ranks_without_group():
    assert not dist.is_initialized()
    assert bench.max_over_ranks(7.5) == 7.5
    assert bench.job_throughput(250.0, 1) == pytest.approx(4.0)


def test_reference_arm_rank_above_zero_exits_quietly(monkeypatch, capsys):
    """Under torchrun the reference arm runs (and prints) on rank 0 only; other ranks return."""
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    bench.run_reference(bench.parse())
    assert capsys.readouterr().out == ""

