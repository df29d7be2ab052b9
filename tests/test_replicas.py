"""The N > 1 path of bench.py on CPU: two gloo ranks, as torchrun launches
them (RANK / WORLD_SIZE / MASTER_ADDR=127.0.0.1).  The imaging path does not
shard (ranks are independent replicas); what is shared is the timing rule --
every rank reports the slowest rank's time, and the whole-job value counts
every replica's samples -- and the reference arm's rule that only rank 0
works.  No GPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, dist, torch, "cpu")
        value = bench.job_throughput(1.0e6, world, ms)
        # the reference arm: ranks other than 0 return without work
        args = type("A", (), {"config": "mid", "ref_baselines": 4, "steps": 1, "warmup": 3, "channels": 1,
                              "hours": 8.0})()
        ref = bench.run_reference(args, rank, world) if rank != 0 else None
        dist.barrier()
        out[rank] = (ms, value, ref)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_slowest_time():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        for p in procs:
            if p.is_alive():
                p.kill()
                pytest.fail("rank did not finish")
            assert p.exitcode == 0
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank in range(world):
        ms, value, ref = res[rank]
        assert ms == 15.0                                   # the slowest rank's time on every rank
        assert value == pytest.approx(1.0e6 * world / 15e-3)
    assert res[1][2] is None                                # rank 1 of the reference arm did no work


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, 1, None, None, "cpu") == 12.5
    assert bench.job_throughput(2.0e6, 1, 20.0) == pytest.approx(1.0e8)
