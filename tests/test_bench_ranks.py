"""The multi-GPU bench path is replicas (each rank sorts its own array); its
host logic — the job's time is the slowest rank's, its correctness every
rank's, its throughput all ranks' keys — runs here on two gloo ranks on CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 20.0][rank]
        ok = rank == 0  # rank 1 reports a failed check
        got_ms, got_ok = bench.reduce_over_ranks(torch, dist, ms, ok, "cpu")
        dist.barrier()
        out[rank] = (got_ms, got_ok)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_every_check():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (20.0, False)


def test_whole_job_throughput_counts_every_rank():
    import bench

    assert bench.whole_job_gkeys(1, 1 << 28, 5.0) == pytest.approx((1 << 28) / 5e-3 / 1e9)
    assert bench.whole_job_gkeys(8, 1 << 28, 5.0) == pytest.approx(8 * bench.whole_job_gkeys(1, 1 << 28, 5.0))


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.reduce_over_ranks(torch, None, 3.0, True, "cpu") == (3.0, True)
