"""The N > 1 path of the benchmark on CPU: two ranks over gloo (127.0.0.1).

The transform does not shard in this workload; several GPUs run independent
replicas.  What the ranks share is host logic: distinct inputs per rank,
the step time as the maximum over ranks, the whole-job rate, and the
reference arm running on rank 0 alone.  Those pieces run here with a gloo
process group of two CPU ranks."""
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
    import datetime
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank reports a different step time; all see the slowest
        t = bench.max_over_ranks(dist, torch, 0.5 + rank, "cpu")
        rate = bench.whole_job_rate(world, 12, t)
        seed = bench.rank_seed(rank)
        # the reference arm works on rank 0 only: other ranks return at once
        ref = bench.run_reference_arm(None, rank) if rank != 0 else "skipped"
        out[rank] = (t, rate, seed, ref)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_timing_and_rate():
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for rank in (0, 1):
        t, rate, seed, ref = res[rank]
        assert t == pytest.approx(1.5)                 # max of 0.5 and 1.5
        assert rate == pytest.approx(2 * 12 / 1.5)     # whole-job sets per second
    assert res[0][2] != res[1][2]                      # replicas transform distinct inputs
    assert res[1][3] is None                           # no reference work on rank 1


def test_single_process_helpers():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, torch, 0.25, "cpu") == 0.25
    assert bench.whole_job_rate(1, 12, 0.75) == pytest.approx(16.0)


def test_clock_summary_covers_the_marked_window_only():
    # the sampler runs for the whole benchmark; only the samples between
    # mark() and end() describe the timed region, and a throttle reason that
    # is active there is reported
    sys.path.insert(0, ROOT)
    import bench
    clk = bench.ClockSampler(0)
    idle = "0, 345, 1965, 120.5, 0x0, Not Active, Not Active, Not Active, Not Active"
    busy = "0, 1965, 1965, 980.0, 0x0, Not Active, Not Active, Not Active, Not Active"
    capped = "0, 1800, 1965, 1000.0, 0x4, Not Active, Not Active, Not Active, Active"
    hot = "0, 1200, 1965, 700.0, 0x40, Not Active, Not Active, Active, Not Active"
    clk.lines = [idle, idle, hot]
    clk.mark()
    clk.lines += [busy, capped, busy]
    clk.end()
    clk.lines += [idle, hot]
    s = clk.summary()
    assert s["samples"] == 3
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    clk.mark()
    clk.lines += ["garbage", "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    clk.end()
    assert clk.summary()["samples"] == 0
