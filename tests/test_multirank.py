"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process
each, rendezvous on 127.0.0.1), as `torchrun --nproc-per-node 2 bench.py`
runs them on two GPUs.  The path runs independent replicas (no collective on
the data path): the only exchanges are the barrier and the max of the timed
seconds over the ranks, and the whole-job rate counts every rank's nodes."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        seconds = [0.25, 0.75][rank]  # rank 1 is the slow one
        dist.barrier()
        slowest = bench.max_over_ranks(torch, dist, seconds, device="cpu")
        out[rank] = (slowest, bench.job_rate(world, 1000, 10, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_count_every_replica():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert out[0] == out[1]
    slowest, rate = out[0]
    assert slowest == 0.75
    assert rate == pytest.approx(world * 1000 * 10 / 0.75 / 1e6)


def test_one_rank_needs_no_process_group():
    assert bench.max_over_ranks(torch, None, 1.5) == 1.5


def test_reference_arm_runs_on_rank_zero_only(capsys):
    class Args:
        n, steps, ref_procs = 8, 1, 1
    bench.run_reference(Args(), rank=1, world=2)
    assert capsys.readouterr().out == ""
