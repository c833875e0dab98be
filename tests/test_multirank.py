"""The multi-GPU host logic of bench.py on two CPU ranks (gloo): every
rank gets the slowest rank's time, the whole-job rate is the replicas'
aggregate over that time, and the reference arm does its work on rank 0
only.  (The path is replicas only: one independent mesh per GPU, no
data-path collective.)"""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slow = bench.max_over_ranks(10.0 + rank, world)          # rank 1 is the slow one
        rate = bench.aggregate_rate(1000, slow / 1e3, world)      # 1000 units per rank in `slow` ms
        calls = []

        class Args:
            cpu_procs, cpu_sample_n, warmup, steps, gpus, n = 1, 4, 1, 1, world, 4

        if rank != 0:
            bench.run_reference_arm(Args, rank, world)            # returns without work
            calls.append("none")
        out[rank] = (slow, rate, calls)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_aggregate():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    assert out[0][0] == out[1][0] == 11.0
    assert abs(out[0][1] - 2 * 1000 / 0.011) < 1e-6
    assert out[1][2] == ["none"]
