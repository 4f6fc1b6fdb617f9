"""The bench's multi-GPU aggregation (one process per GPU, replicas): every
rank's timed region ends in a max-over-ranks reduction and the whole-job rate
counts all ranks' units over the slowest rank's time.  Exercised here with two
gloo ranks on the CPU."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert bench._rank_env()[:2] == (rank, world)
        # rank 1 is the slower one in the first value, rank 0 in the second
        mine = [1.0 + rank, 5.0 - rank]
        out[rank] = bench.max_over_ranks(dist, mine, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    with mp.get_context("spawn").Manager() as mgr:  # no fork of a process that already runs threads
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        got = dict(out)
    assert got[0] == got[1] == [2.0, 5.0]


def test_whole_job_rate_and_single_process_path():
    import bench

    assert bench.max_over_ranks(None, [3, 4.5], "cpu") == [3.0, 4.5]
    # 4 ranks, 1e9 units each, slowest rank 2 s -> 2e9 units/s for the job
    assert bench.whole_job_rate(4, 1e9, 2.0) == pytest.approx(2e9)


def test_roofline_inputs_of_the_bench_line():
    # traffic: the DRAM bytes per launch that the committed ncu summary records
    import bench

    assert bench.profile_traffic("k_sweep_rmat22.md") == 416051200.0
    assert bench.profile_traffic("no_such_profile.md") is None
    peak, kind = bench.measured_peaks()
    assert peak > 0 and kind in ("measured", "fallback")
