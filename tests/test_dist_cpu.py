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


# ---------------------------------------------------------------------------
# One transform over several ranks (sharp_b200.distributed): the ring pairs
# are split between two gloo ranks, each rank runs its share with the
# reference library standing in for its GPU, and the partial a_lm are summed
# by the collective.  Every rank's result must equal the single-process
# reference transform.
# ---------------------------------------------------------------------------
def _ref_subset(ref):
    import numpy as np

    def subset(g, pairs):
        gi = g.ptr.contents
        rings = []
        for i in pairs:
            pr = gi.pair[i]
            rings.append(pr.r1)
            if pr.r2.nph > 0:
                rings.append(pr.r2)
        f = lambda k, t: np.array([getattr(r, k) for r in rings], t)  # noqa: E731
        return ref.general(f("nph", np.int32), f("ofs", np.intp), f("stride", np.int32),
                           f("phi0", np.float64), f("theta", np.float64), f("weight", np.float64))
    return subset


def _split_rank_main(rank, world, port, out):
    import datetime
    import numpy as np
    os.environ["OMP_NUM_THREADS"] = "2"
    for sub in ("planck-levels_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import ref
    import sharp_b200 as sb
    from sharp_b200 import distributed as sd
    from helpers import rel_l2, uniform_alm
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        nside, lmax = 32, 64
        g, a = ref.healpix(nside), ref.triangular(lmax, lmax)
        npix = 12 * nside * nside
        res = {}
        for spin in (0, 2):
            nc = 1 if spin == 0 else 2
            split = sd.RingSplit(g, lmax, lmax, spin, rank, world, subset=_ref_subset(ref))
            res[f"imbalance{spin}"] = split.imbalance()
            res[f"npairs{spin}"] = len(split.pairs)
            alms = [uniform_alm(lmax, seed=30 + i, spin=spin) for i in range(nc)]
            # synthesis: this rank's rings, and the whole map with gather=True
            full = [np.zeros(npix) for _ in range(nc)]
            ref.execute(1, spin, [x.copy() for x in alms], full, g, a, 1, sb.SHARP_DP)
            mine = [np.zeros(npix) for _ in range(nc)]
            sd.execute(split, 1, spin, [x.copy() for x in alms], mine, a, 1, sb.SHARP_DP,
                       run=ref.execute)
            gi = split.local.ptr.contents
            idx = np.concatenate([r.ofs + np.arange(r.nph) for i in range(gi.npairs)
                                  for r in (gi.pair[i].r1, gi.pair[i].r2) if r.nph > 0])
            res[f"synth_local{spin}"] = max(rel_l2(x[idx], y[idx]) for x, y in zip(mine, full))
            res[f"synth_other_zero{spin}"] = all(
                np.count_nonzero(x) <= len(idx) for x in mine)
            got = [np.full(npix, 5.0) for _ in range(nc)]
            sd.execute(split, 1, spin, [x.copy() for x in alms], got, a, 1, sb.SHARP_DP,
                       run=ref.execute, gather=True)
            res[f"synth_gather{spin}"] = max(rel_l2(x, y) for x, y in zip(got, full))
            # analysis: complete a_lm on every rank, with and without SHARP_ADD,
            # and the unweighted transpose (SHARP_Yt)
            want = [np.zeros_like(alms[0]) for _ in range(nc)]
            ref.execute(0, spin, want, [x.copy() for x in full], g, a, 1, sb.SHARP_DP)
            got = [np.zeros_like(alms[0]) for _ in range(nc)]
            sd.execute(split, 0, spin, got, [x.copy() for x in full], a, 1, sb.SHARP_DP,
                       run=ref.execute)
            res[f"anal{spin}"] = max(rel_l2(x, y) for x, y in zip(got, want))
            got = [x.copy() for x in alms]
            sd.execute(split, 0, spin, got, [x.copy() for x in full], a, 1,
                       sb.SHARP_DP | sb.SHARP_ADD, run=ref.execute)
            res[f"anal_add{spin}"] = max(rel_l2(x, y + z) for x, y, z in zip(got, want, alms))
            wt = [np.zeros_like(alms[0]) for _ in range(nc)]
            ref.execute(2, spin, wt, [x.copy() for x in full], g, a, 1, sb.SHARP_DP)
            got = [np.zeros_like(alms[0]) for _ in range(nc)]
            sd.execute(split, 2, spin, got, [x.copy() for x in full], a, 1, sb.SHARP_DP,
                       run=ref.execute)
            res[f"yt{spin}"] = max(rel_l2(x, y) for x, y in zip(got, wt))
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_ring_split_transform_over_two_gloo_ranks():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_split_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for spin in (0, 2):
        assert res[0][f"npairs{spin}"] + res[1][f"npairs{spin}"] == 64   # Nside 32: 63 rings / 2 + 1
        assert res[0][f"npairs{spin}"] > 0 and res[1][f"npairs{spin}"] > 0
        for r in (0, 1):
            d = res[r]
            assert d[f"imbalance{spin}"] < 0.05
            assert d[f"synth_local{spin}"] < 1e-12 and d[f"synth_other_zero{spin}"]
            for k in ("synth_gather", "anal", "anal_add", "yt"):
                assert d[f"{k}{spin}"] < 1e-12, (r, k, spin, d[f"{k}{spin}"])


def test_ring_partition_balances_healpix_pairs():
    for sub in ("planck-levels_b200",):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import numpy as np
    import sharp_b200 as sb
    from sharp_b200 import distributed as sd
    g = sb.Geometry.healpix(256)
    costs = sd.pair_costs(g, 512, 512, 2)
    for world in (2, 4, 8):
        parts = sd.partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(g.npairs))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) / np.mean(loads) - 1 < 0.01
