"""The replicas path of bench.py on CPU: two gloo ranks, the way torchrun launches it on two GPUs.

The encode does not shard (one material per GPU); what runs across ranks is host logic only: the barrier around the
timed steps, the max over ranks of the measured times, the whole-job value over all ranks, and the reference arm,
which runs on rank 0 alone while the other ranks exit 0 without work."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, world, rank)
        dist.barrier()
        # rank r measured 100 + 50 r ms on the device and 300 - 10 r ms end to end
        device_ms, e2e_ms = bench.slowest(world, [100.0 + 50.0 * rank, 300.0 - 10.0 * rank], "cpu")
        out[rank] = (device_ms, e2e_ms, bench.job_value(world, 4.0, 2, device_ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(rank_main, args=(world, free_port(), out), nprocs=world, start_method="spawn", join=True)
    for rank in range(world):
        device_ms, e2e_ms, value = out[rank]
        assert device_ms == 150.0 and e2e_ms == 300.0   # every rank sees the slowest rank's times
        assert value == pytest.approx(2 * 4.0 * 2 / 0.150)


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        config, crop, steps, warmup = 0, 16, 1, 0

    # a rank other than 0 returns at once, before any material is built or any encoder is run
    assert bench.run_reference(Args(), rank=1, world=2) == 0
