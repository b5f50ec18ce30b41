#!/usr/bin/env python
"""Throughput of the spherical-harmonic transform engine on the headline
workload: alm2map + map2alm round trips of a temperature+polarisation set
(one spin-0 job T and one spin-2 job E,B -> Q,U per direction, as
Healpix_cxx alm2map_pol / map2alm_pol do) on a HEALPix Nside=2048 map with
lmax = mmax = 4096.

Two forms are measured in the same run:
  * mixed (headline): a batch of B independent T+QU sets per step, every
    sharp_execute job with ntrans = B and SHARP_MIXED (exact-integer
    tensor-core Legendre contraction where the library has one, FP64
    elsewhere).  value = round trips (sets) per second over all ranks; the
    line carries the relative L2 error of the batch's outputs against the
    FP64 path on the same inputs.
  * fp64: the plain FP64 drop-in, one set per step (ntrans = 1).
One step = T+QU alm2map followed by T+QU map2alm for each set of the step.
``value`` has the inputs resident in HBM; ``e2e`` is the same metric through
the C ABI with pinned host buffers, so every step includes the host<->device
copies: one sharp_b200_execute_batch call per step holding the round trip
(T and QU alm2map, then T and QU map2alm of the maps just written to host
memory), with the figures for one batch call per direction and for four
sharp_execute calls beside it.  N>1 runs independent replicas (the transform does
not shard across GPUs in this workload).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B]
                    [--form mixed|fp64] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "planck-levels_b200"), os.path.join(ROOT, "oracle"),
                os.path.join(ROOT, "tests")]

METRIC = "alm2map+map2alm /s at Nside 2048, lmax 4096: mixed vs FP64 GPU at <=1e-6 err"
UNIT = "transforms/s"
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nside", type=int, default=2048)
    ap.add_argument("--lmax", type=int, default=4096)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--form", default="mixed", choices=["mixed", "fp64"],
                    help="headline form: batched SHARP_MIXED or the FP64 drop-in")
    ap.add_argument("--batch", type=int, default=12, help="T+QU sets per step (mixed form)")
    ap.add_argument("--fp64-steps", type=int, default=4,
                    help="timed steps of the FP64 drop-in companion measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-only", action="store_true",
                    help="run warm-up and timed steps only (for ncu launch lists)")
    return ap.parse_args()


def inputs(lmax, seed=7):
    import numpy as np
    from helpers import cl_spectrum, random_alm
    cl = cl_spectrum(lmax, beam_arcmin=5.0)
    rng = np.random.default_rng(seed)
    t = random_alm(lmax, cl=cl, rng=rng)
    e = random_alm(lmax, cl=0.1 * cl, rng=rng)
    b = random_alm(lmax, cl=0.01 * cl, rng=rng)
    return t, e, b


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = 0
        self.last = None

    def mark(self):
        """Only samples taken after this call (and before end()) enter the
        summary.  The sampler runs from the start of the benchmark: the first
        nvidia-smi on a freshly reset GPU holds the driver for a while, and
        a workspace allocation waiting on it must not fall into a timed
        region."""
        self.first = len(self.lines)
        self.last = None

    def end(self):
        self.last = len(self.lines)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:self.last]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def fp64_gemm_peak(torch):
    """Measured FP64 peak on this GPU: cuBLAS DGEMM 8192^3 (best of 5)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def dram_traffic_from_profiles(family):
    """Per-launch DRAM bytes of a kernel family from its committed ncu
    summary (line 'dram_bytes_per_launch: <int>'), else None."""
    name = TRAFFIC_FILE.get(family)
    if not name:
        return None
    try:
        for ln in open(os.path.join(ROOT, "profiles", name)):
            if ln.startswith("dram_bytes_per_launch:"):
                return int(float(ln.split(":")[1]))
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# reference arm (CPU, libsharp built from the reference sources)
# ---------------------------------------------------------------------------
def reference_round_trip(ref, geom, ainfo, t, e, b, npix):
    import numpy as np
    DP = 1 << 4
    mt = np.zeros(npix); mq = np.zeros(npix); mu = np.zeros(npix)
    t0 = time.perf_counter()
    ref.execute(1, 0, [t], [mt], geom, ainfo, 1, DP)
    ref.execute(1, 2, [e, b], [mq, mu], geom, ainfo, 1, DP)
    ot = np.zeros_like(t); oe = np.zeros_like(e); ob = np.zeros_like(b)
    ref.execute(0, 0, [ot], [mt], geom, ainfo, 1, DP)
    ref.execute(0, 2, [oe, ob], [mq, mu], geom, ainfo, 1, DP)
    return time.perf_counter() - t0


def run_reference_arm(args, rank):
    if rank != 0:
        return None
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsharp_ref.so not built"}))
        return None
    t, e, b = inputs(args.lmax)
    geom = ref.healpix(args.nside)
    ainfo = ref.triangular(args.lmax, args.lmax)
    npix = 12 * args.nside ** 2
    for _ in range(args.warmup):
        reference_round_trip(ref, geom, ainfo, t, e, b, npix)
    times = [reference_round_trip(ref, geom, ainfo, t, e, b, npix) for _ in range(args.steps)]
    tot = sum(times)
    value = args.steps / tot
    sample = (f"{args.steps} full T+QU round trips (spin-0 + spin-2 alm2map and map2alm, FP64) "
              f"at Nside {args.nside}, lmax {args.lmax}, reference libsharp with OpenMP")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"T+QU alm2map+map2alm, HEALPix Nside {args.nside}, "
                                   f"lmax=mmax={args.lmax}, spin 0+2, FP64",
                       "nside": args.nside, "lmax": args.lmax, "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return line


def cpu_baseline(args):
    """Reference libsharp on all host cores, one T+QU round trip (bounded)."""
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    import ref
    if not ref.available():
        return None
    t, e, b = inputs(args.lmax)
    geom = ref.healpix(args.nside)
    ainfo = ref.triangular(args.lmax, args.lmax)
    npix = 12 * args.nside ** 2
    # small warm-up (spawns the OpenMP team, runs libsharp's nv autotuner)
    g2, a2 = ref.healpix(64), ref.triangular(128, 128)
    ts, es, bs = inputs(128)
    reference_round_trip(ref, g2, a2, ts, es, bs, 12 * 64 * 64)
    dt = reference_round_trip(ref, geom, ainfo, t, e, b, npix)
    return {"value": 1.0 / dt, "unit": UNIT, "cores": int(os.environ.get("OMP_NUM_THREADS", cores)),
            "kind": "reference",
            "sample": f"1 full T+QU round trip (spin-0 + spin-2 alm2map and map2alm, FP64) at "
                      f"Nside {args.nside}, lmax {args.lmax}: reference libsharp with OpenMP, "
                      f"{dt:.2f} s"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
FAMILIES = ("legendre_synth", "legendre_anal", "mixed_synth_spin0", "mixed_synth_spin",
            "mixed_anal_spin0", "mixed_anal_spin", "ring_synth", "ring_anal", "stage_alm",
            "scatter_alm", "mixed_image")
LEGENDRE = FAMILIES[:6]
# profile summary holding 'dram_bytes_per_launch: <int>' for each family
TRAFFIC_FILE = {"mixed_anal_spin": "mixed_anal_spin2_nside2048.txt",
                "mixed_anal_spin0": "mixed_anal_spin0_nside2048.txt",
                "mixed_synth_spin": "mixed_synth_spin2_nside2048.txt",
                "mixed_synth_spin0": "mixed_synth_spin0_nside2048.txt",
                "legendre_anal": "legendre_anal_fp64_nside2048.txt",
                "legendre_synth": "legendre_synth_fp64_nside2048.txt"}


class Sets:
    """B independent T+QU sets resident on the device: a_lm inputs, maps,
    round-trip a_lm outputs (float64 views of complex128 a_lm)."""

    def __init__(self, sb, torch, np, dev, lmax, npix, nalm, count, seed0):
        self.count = count
        self.host = [inputs(lmax, seed=seed0 + i) for i in range(count)]

        def dalm(x):
            return torch.from_numpy(x.view(np.float64).copy()).to(dev)

        self.a = [[dalm(x) for x in h] for h in self.host]           # (t, e, b)
        self.m = [[torch.zeros(npix, dtype=torch.float64, device=dev) for _ in range(3)]
                  for _ in range(count)]                               # (T, Q, U)
        self.o = [[torch.zeros(2 * nalm, dtype=torch.float64, device=dev) for _ in range(3)]
                  for _ in range(count)]

    def step(self, sb, geom, ainfo, n, flags, ops=None):
        r = range(n)
        ops = {} if ops is None else ops
        ops["s0_synth"] = sb.execute_device(sb.SHARP_ALM2MAP, 0, [self.a[i][0] for i in r],
                                            [self.m[i][0] for i in r], geom, ainfo, n, flags)
        ops["s2_synth"] = sb.execute_device(
            sb.SHARP_ALM2MAP, 2, [x for i in r for x in self.a[i][1:]],
            [x for i in r for x in self.m[i][1:]], geom, ainfo, n, flags)
        ops["s0_anal"] = sb.execute_device(sb.SHARP_MAP2ALM, 0, [self.o[i][0] for i in r],
                                           [self.m[i][0] for i in r], geom, ainfo, n, flags)
        ops["s2_anal"] = sb.execute_device(
            sb.SHARP_MAP2ALM, 2, [x for i in r for x in self.o[i][1:]],
            [x for i in r for x in self.m[i][1:]], geom, ainfo, n, flags)
        return ops


def max_over_ranks(dist, torch, value, device):
    """The largest value over all ranks (the slowest rank's time), or the
    value itself without a process group."""
    if not dist:
        return value
    tt = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def rank_seed(rank):
    """Seed of the first input set of a rank: replicas transform distinct
    inputs."""
    return 7 + 1000 * rank


def whole_job_rate(world, per_rank_units, step_s):
    """Units processed by all ranks per second when every rank processes
    per_rank_units in step_s (the max over ranks)."""
    return world * per_rank_units / step_s


def timed(torch, lib, stream, fn, steps, warmup, dist, clk=None):
    """Device time per step (CUDA events on the launching stream, barrier +
    synchronize on both sides), launch count and per-family kernel time."""
    lib.sharp_b200_profile(1)   # warm-up runs with the same event instrumentation
    for i in range(warmup):
        fn()
        if i == 0:
            # the first step after a synchronize grows the library's workspace
            # pool once (its buffers then no longer fit the chunks the first
            # step left); let that happen here rather than in the timed steps
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = lib.sharp_b200_kernel_launches()
    # per-family totals of the warm-up, subtracted below (the instrumentation
    # stays as it is across the start of the timed region)
    base = {}
    for name in FAMILIES:
        n = C.c_ulonglong(0)
        base[name] = (lib.sharp_b200_profile_ms(name.encode(), C.byref(n)), n.value)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    if clk:
        clk.mark()
    # a full Python garbage collection costs ~0.4 s of host time in this
    # process: run it here and keep the collector off while timing
    gc.collect()
    gc.disable()
    host = []
    evs[0].record(stream)
    for i in range(steps):
        h0 = time.perf_counter()
        fn()
        host.append(round((time.perf_counter() - h0) * 1e3, 2))
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    gc.enable()
    if clk:
        clk.end()
    if dist:
        dist.barrier()
    launches = lib.sharp_b200_kernel_launches() - l0
    fam = {}
    for name in FAMILIES:
        n = C.c_ulonglong(0)
        ms = lib.sharp_b200_profile_ms(name.encode(), C.byref(n))
        if n.value > base[name][1]:
            fam[name] = (ms - base[name][0], n.value - base[name][1])
    lib.sharp_b200_profile(0)
    step_s = evs[0].elapsed_time(evs[-1]) * 1e-3 / steps
    per_step = [round(evs[i].elapsed_time(evs[i + 1]), 2) for i in range(steps)]
    step_s = max_over_ranks(dist, torch, step_s, "cuda")
    # per_step: device time between the step events; host: time the host
    # took to enqueue each step (a step whose device time exceeds its kernels'
    # sum by more than its host time waited on something outside the library)
    return step_s, launches, fam, {"device": per_step, "host_enqueue": host}


def rel(torch, a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # CPU arm: rank 0 alone, other ranks exit without work
        run_reference_arm(args, rank)
        return

    import numpy as np
    import torch
    import sharp_b200 as sb

    torch.cuda.set_device(local)
    # clocks are sampled from here to the end; the timed regions mark theirs
    with ClockSampler(local) as clk:
        run_ours(args, world, rank, local, clk, np, torch, sb)


def run_ours(args, world, rank, local, clk, np, torch, sb):
    """Our arm: timed device steps, the FP64 companion and the e2e run."""
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    nside, lmax = args.nside, args.lmax
    npix = 12 * nside * nside
    nalm = sb.nalm_triangular(lmax)
    geom = sb.Geometry.healpix(nside)
    ainfo = sb.AlmInfo.triangular(lmax)
    dev = torch.device("cuda", local)
    mixed = args.form == "mixed"
    B = max(1, args.batch) if mixed else 1
    DP = sb.SHARP_DP
    flags = DP | (sb.SHARP_MIXED if mixed else 0)
    sets = Sets(sb, torch, np, dev, lmax, npix, nalm, B, seed0=rank_seed(rank))

    lib = sb.lib()
    lib.sharp_b200_kernel_launches.restype = C.c_ulonglong
    lib.sharp_b200_profile_ms.restype = C.c_double
    lib.sharp_b200_profile_ms.argtypes = [C.c_char_p, C.POINTER(C.c_ulonglong)]
    stream = torch.cuda.current_stream()

    ops = {}
    step_s, launches, fam, per_step = timed(torch, lib, stream,
                                            lambda: sets.step(sb, geom, ainfo, B, flags, ops),
                                            args.steps, args.warmup, dist, clk)
    if args.profile_only:
        if dist:
            dist.destroy_process_group()
        return
    value = whole_job_rate(world, B, step_s)
    # outputs of every set of the headline batch (compared with FP64 below)
    head_all = [[x.clone() for x in sets.m[i] + sets.o[i]] for i in range(B)]
    head_out = head_all[0]

    # the FP64 drop-in on set 0 (ntrans = 1): companion number and the error
    # reference for the mixed outputs
    fp64_ops = {}
    fp64_s, fp64_launches, fp64_fam, _ = timed(
        torch, lib, stream, lambda: sets.step(sb, geom, ainfo, 1, DP, fp64_ops),
        args.fp64_steps if mixed else args.steps, 2, dist)
    # error of every set of the batch: the batch's round-trip outputs
    # (mixed) against one untimed FP64 pass over all sets on the same inputs
    err = {"maps": 0.0, "alms": 0.0, "sets": B}
    if mixed:
        sets.step(sb, geom, ainfo, B, DP)
        torch.cuda.synchronize()
        per_set = []
        for i in range(B):
            ref_i = sets.m[i] + sets.o[i]
            em = max(rel(torch, head_all[i][j], ref_i[j]) for j in range(3))
            ea = max(rel(torch, head_all[i][j], ref_i[j]) for j in range(3, 6))
            per_set.append([em, ea])
        err = {"maps": max(x[0] for x in per_set), "alms": max(x[1] for x in per_set),
               "sets": B, "per_set_maps_alms": per_set,
               "what": "max relative L2 error over the T,Q,U maps and the T,E,B round-trip "
                       "a_lm of each set, mixed batch against FP64 on the same input a_lm"}
    del head_all         # set 0's outputs stay referenced for the host-path check

    # end-to-end through sharp_execute with pinned host buffers, the same
    # batch and flags as the headline
    def pinned(n, dtype):
        return torch.empty(n, dtype=dtype, pin_memory=True).numpy()

    try:
        import psutil
        avail = psutil.virtual_memory().available
    except ImportError:
        avail = 0
    need = B * 3 * (npix * 8 + 2 * nalm * 16)
    # distinct host buffers when host memory allows (the ranks of this node
    # allocate theirs at the same time)
    local_world = max(1, int(os.environ.get("LOCAL_WORLD_SIZE", str(world))))
    nh = B if avail > 4 * need * local_world else 1
    h_alm = [[pinned(nalm, torch.complex128) for _ in range(3)] for _ in range(nh)]
    h_map = [[pinned(npix, torch.float64) for _ in range(3)] for _ in range(nh)]
    h_out = [[pinned(nalm, torch.complex128) for _ in range(3)] for _ in range(nh)]
    for i in range(nh):
        for j in range(3):
            h_alm[i][j][:] = sets.host[i][j]
    hs = [i % nh for i in range(B)]

    def host_step():
        sb.execute(sb.SHARP_ALM2MAP, 0, [h_alm[i][0] for i in hs], [h_map[i][0] for i in hs],
                   geom, ainfo, B, flags)
        sb.execute(sb.SHARP_ALM2MAP, 2, [x for i in hs for x in h_alm[i][1:]],
                   [x for i in hs for x in h_map[i][1:]], geom, ainfo, B, flags)
        sb.execute(sb.SHARP_MAP2ALM, 0, [h_out[i][0] for i in hs], [h_map[i][0] for i in hs],
                   geom, ainfo, B, flags)
        sb.execute(sb.SHARP_MAP2ALM, 2, [x for i in hs for x in h_out[i][1:]],
                   [x for i in hs for x in h_map[i][1:]], geom, ainfo, B, flags)

    def host_time(fn, steps):
        # two untimed steps: every host-array call ends with a synchronize,
        # and the second such step is where the workspace pool takes its
        # steady size
        for _ in range(2):
            fn()
        if dist:
            dist.barrier()
        gc.collect()
        gc.disable()
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        dt = (time.perf_counter() - t0) / steps
        gc.enable()
        return max_over_ranks(dist, torch, dt, dev)

    # the same step through the batch entry: the four jobs of the round trip
    # in one call (the map2alm jobs read the maps the alm2map jobs write into
    # host memory; the library orders those copies), so the host<->device
    # copies overlap the compute across all jobs: one fill and one drain per
    # step
    synth_jobs = [
        (sb.SHARP_ALM2MAP, 0, [h_alm[i][0] for i in hs], [h_map[i][0] for i in hs],
         geom, ainfo, B, flags),
        (sb.SHARP_ALM2MAP, 2, [x for i in hs for x in h_alm[i][1:]],
         [x for i in hs for x in h_map[i][1:]], geom, ainfo, B, flags)]
    anal_jobs = [
        (sb.SHARP_MAP2ALM, 0, [h_out[i][0] for i in hs], [h_map[i][0] for i in hs],
         geom, ainfo, B, flags),
        (sb.SHARP_MAP2ALM, 2, [x for i in hs for x in h_out[i][1:]],
         [x for i in hs for x in h_map[i][1:]], geom, ainfo, B, flags)]

    def host_step_batch():
        sb.execute_batch(synth_jobs + anal_jobs)

    # the same with one batch call per direction
    def host_step_directions():
        sb.execute_batch(synth_jobs)
        sb.execute_batch(anal_jobs)

    e2e_exec_s = host_time(host_step, args.e2e_steps)
    e2e_dir_s = host_time(host_step_directions, args.e2e_steps)
    e2e_s = host_time(host_step_batch, args.e2e_steps)

    # the FP64 drop-in end to end: one T+QU set per step through
    # sharp_execute with host arrays, as alm2map_pol / map2alm_pol call it
    def host_step_fp64():
        sb.execute(sb.SHARP_ALM2MAP, 0, [h_alm[0][0]], [h_map[0][0]], geom, ainfo, 1, DP)
        sb.execute(sb.SHARP_ALM2MAP, 2, h_alm[0][1:], h_map[0][1:], geom, ainfo, 1, DP)
        sb.execute(sb.SHARP_MAP2ALM, 0, [h_out[0][0]], [h_map[0][0]], geom, ainfo, 1, DP)
        sb.execute(sb.SHARP_MAP2ALM, 2, h_out[0][1:], h_map[0][1:], geom, ainfo, 1, DP)

    fp64_e2e_s = host_time(host_step_fp64, args.e2e_steps)
    # the check run: one round-trip batch call from cleared map and output
    # buffers, so the map2alm jobs can only see maps this call wrote
    for i in range(nh):
        for j in range(3):
            h_map[i][j][:] = 0.0
            h_out[i][j][:] = 0.0
    host_step_batch()
    h2d = B * (3 * nalm * 16 + 3 * npix * 8)
    d2h = B * (3 * npix * 8 + 3 * nalm * 16)
    t_in = sets.host[0][0]
    # set 0 through the host batch against the device-resident step: maps
    # (written by the alm2map jobs) and round-trip a_lm (map2alm of those maps)
    def _rel(dev_t, host, cpx):
        d = dev_t.cpu().numpy()
        d = d.view(np.complex128) if cpx else d
        return float(np.linalg.norm(d - host) / np.linalg.norm(host))
    api_err = max([_rel(head_out[j], h_map[0][j], False) for j in range(3)] +
                  [_rel(head_out[3 + j], h_out[0][j], True) for j in range(3)])
    rt_err = float(np.linalg.norm(h_out[0][0] - t_in) / np.linalg.norm(t_in))

    # roofline of the dominant Legendre kernel family
    dom = max((f for f in LEGENDRE if f in fam), key=lambda k: fam[k][0])
    dom_ms, dom_n = fam[dom]
    roof = roofline(dom, dom_ms, dom_n, ops, B, args.steps, fp64_gemm_peak(torch))
    tot = sum(v[0] for v in fam.values())
    share = {k: round(v[0] / max(1e-9, tot), 4) for k, v in fam.items()}

    form = (f"mixed: batch of {B} sets per step, SHARP_MIXED (int8 tensor-core Legendre "
            f"synthesis and analysis)" if mixed else "fp64 drop-in, one set per step")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+i8" if mixed else "f64", "data": "synthetic",
            "config": {"workload": f"T+QU alm2map+map2alm, HEALPix Nside {nside}, "
                                   f"lmax=mmax={lmax}, spin 0+2, {form}",
                       "nside": nside, "lmax": lmax, "form": args.form, "batch": B,
                       "alm": "a_lm ~ C_l = (l+1)^-2 exp(-l(l+1) sigma^2), sigma 5', E 0.1, B 0.01",
                       "l2": f"inputs larger than L2 (each map {npix * 8 / 1e6:.0f} MB, "
                             f"each a_lm {nalm * 16 / 1e6:.0f} MB)",
                       "parallelism": f"replicas x{world}"},
            "rel_err_vs_fp64": err,
            "fp64_dropin": {"value": world / fp64_s, "unit": UNIT, "ms_per_step": fp64_s * 1e3,
                            "kernel_ms_per_step": {k: round(v[0] / (args.fp64_steps if mixed
                                                                      else args.steps), 3)
                                                   for k, v in fp64_fam.items()},
                            "e2e": {"value": world / fp64_e2e_s, "unit": UNIT,
                                    "steps": args.e2e_steps,
                                    "h2d_bytes_per_step": h2d // B,
                                    "d2h_bytes_per_step": d2h // B,
                                    "what": "one T+QU set per step through sharp_execute with "
                                            "host arrays (four calls, ntrans = 1)"}},
            "e2e": {"value": whole_job_rate(world, B, e2e_s), "unit": UNIT, "steps": args.e2e_steps,
                    "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "host_buffers": "distinct" if nh == B else "shared",
                    "api": "one sharp_b200_execute_batch call per step with host arrays: "
                           "T and QU alm2map, then T and QU map2alm of the maps written "
                           "(a round trip through host memory)",
                    "per_direction": {"value": whole_job_rate(world, B, e2e_dir_s), "unit": UNIT,
                                      "api": "two sharp_b200_execute_batch calls per step "
                                             "(alm2map jobs, then map2alm jobs)"},
                    "sharp_execute": {"value": whole_job_rate(world, B, e2e_exec_s), "unit": UNIT,
                                      "api": "four sharp_execute calls per step (ntrans = B)"}},
            "gpu_launches": int(launches),
            "roofline": roof,
            "kernel_time_share": share,
            "kernel_ms_per_step": {k: round(v[0] / args.steps, 3) for k, v in fam.items()},
            "step_ms": per_step["device"],
            "step_host_enqueue_ms": per_step["host_enqueue"],
            "clocks": clk.summary(),
            "check": {"round_trip_rel_err_no_iteration": rt_err, "device_vs_host_api": api_err}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def roofline(dom, dom_ms, dom_n, ops, B, steps, peak):
    """Achieved FP64 rate of the dominant Legendre family against the
    DGEMM peak measured in the same run, per launch.

    FP64 kernels: the reference's operation count (sharp_execute's opcnt).
    Mixed kernels: the FP64 work their producers execute per (ring pair, l)
    value, the recurrence plus the quantisation of its values: 5 flops at
    spin 0 (DMUL + 2 DFMA) and 12 at spin s (two recurrences of 2 DFMA each
    plus two quantising DFMA); every launch covers all (ring pair, l) values
    of its job.  The contraction itself runs on the int8 tensor pipe."""
    job = {"legendre_synth": ("s0_synth", "s2_synth"), "legendre_anal": ("s0_anal", "s2_anal"),
           "mixed_synth_spin0": ("s0_synth",), "mixed_synth_spin": ("s2_synth",),
           "mixed_anal_spin0": ("s0_anal",), "mixed_anal_spin": ("s2_anal",)}[dom]
    leg = None
    if dom.startswith("mixed"):
        spin2 = dom.endswith("spin")
        values = ops[job[0]] / ((12 + 16 * B) if spin2 else (4 + 4 * B))
        flops_step = values * (12 if spin2 else 5) * dom_n / steps
        what = "mixed-kernel producer FP64 work (recurrence + quantisation), all launches of a step"
        # the algorithmic count (the reference's opcnt of the whole
        # B-transform job, F_leg = triples (12 + 16 B) at spin s, (4 + 4 B) at 0)
        leg = ops[job[0]] / (dom_ms * 1e-3 / steps) / 1e12
    else:
        flops_step = sum(ops[j] for j in job)
        what = "reference operation count"
    achieved = flops_step * steps / (dom_ms * 1e-3) / 1e12
    traffic = dram_traffic_from_profiles(dom)
    out = {"bound": "fp64", "kernel": dom, "achieved": achieved, "peak": peak,
           "unit": "TFLOP/s", "frac": achieved / peak, "work": what,
           "peak_source": "cuBLAS DGEMM 8192^3 measured in this run "
                          "(MEASURED_PEAKS.json holds no FP64 figure)",
           "flops_per_launch": flops_step * steps / max(dom_n, 1),
           "ms_per_launch": dom_ms / max(dom_n, 1),
           "launches_per_step": dom_n / steps,
           "traffic": traffic,
           "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per launch at "
                              "Nside 512 / lmax 1024, scaled x16 to Nside 2048 / lmax 4096 "
                              "(phase bytes grow with rings x (mmax+1), coefficient and a_lm "
                              "bytes with lmax^2)") if traffic else None}
    if leg is not None:
        out["fp64_equivalent"] = {"achieved": leg, "frac": leg / peak,
                                  "work": "F_leg of the job (reference opcnt, 12 + 16 ntrans "
                                          "per (l, m, pair) at spin s, 4 + 4 ntrans at spin 0) "
                                          "over the family's time"}
    return out


if __name__ == "__main__":
    main()
