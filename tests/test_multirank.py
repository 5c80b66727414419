"""The multi-GPU path of bench.py on CPU: two gloo ranks (replicas, no data
exchange; the only collective is the max-over-ranks of the step time), and the
reference arm's rank behaviour under torchrun (rank 0 alone runs)."""

import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, torch.device("cpu"))
        out[rank] = (ms, bench.job_steps_per_s(world, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        ms, value = out[r]
        assert ms == 15.0  # the slowest rank sets the step time
        assert value == pytest.approx(world * 1000.0 / 15.0)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, None, torch.device("cpu")) == 3.5
    assert bench.job_steps_per_s(1, 4.0) == 250.0


def test_reference_arm_other_ranks_do_nothing(capsys):
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    args = argparse.Namespace(steps=1, warmup=3, gpus=2)
    bench.run_reference(args, rank=1, world=2)
    assert capsys.readouterr().out == ""
