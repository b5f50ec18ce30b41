#!/usr/bin/env python
"""Throughput of the spherical-harmonic transform engine on the headline
workload: alm2map + map2alm round trips of a temperature+polarisation set
(one spin-0 job T and one spin-2 job E,B -> Q,U per direction, as
Healpix_cxx alm2map_pol / map2alm_pol do) on a HEALPix Nside=2048 map with
lmax = mmax = 4096, FP64.

One step = T+QU alm2map followed by T+QU map2alm.  ``value`` is round trips
per second over all ranks with inputs resident in HBM; ``e2e`` is the same
metric through the C ABI (sharp_execute) with pinned host buffers, so every
step includes the host<->device copies.  N>1 runs independent replicas (the
transform does not shard across GPUs in this workload).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
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
    ap.add_argument("--e2e-steps", type=int, default=3)
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
        for ln in self.lines:
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


def dram_traffic_from_profiles():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (line 'dram_bytes_per_launch: <int>'), else None."""
    path = os.path.join(ROOT, "profiles", "legendre_synth_nside2048.txt")
    try:
        for ln in open(path):
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
    t, e, b = inputs(lmax, seed=7 + rank)
    dev = torch.device("cuda", local)

    def dalm(x):
        return torch.from_numpy(x.view(np.float64).copy()).to(dev)

    at, ae, ab = dalm(t), dalm(e), dalm(b)
    mt, mq, mu = (torch.zeros(npix, dtype=torch.float64, device=dev) for _ in range(3))
    ot, oe, ob = (torch.zeros(2 * nalm, dtype=torch.float64, device=dev) for _ in range(3))
    DP = sb.SHARP_DP
    flops = {}

    def step():
        flops["s0_synth"] = sb.execute_device(sb.SHARP_ALM2MAP, 0, [at], [mt], geom, ainfo, 1, DP)
        flops["s2_synth"] = sb.execute_device(sb.SHARP_ALM2MAP, 2, [ae, ab], [mq, mu], geom, ainfo,
                                              1, DP)
        flops["s0_anal"] = sb.execute_device(sb.SHARP_MAP2ALM, 0, [ot], [mt], geom, ainfo, 1, DP)
        flops["s2_anal"] = sb.execute_device(sb.SHARP_MAP2ALM, 2, [oe, ob], [mq, mu], geom, ainfo,
                                             1, DP)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    lib = sb.lib()
    lib.sharp_b200_kernel_launches.restype = C.c_ulonglong
    lib.sharp_b200_profile_ms.restype = C.c_double
    lib.sharp_b200_profile_ms.argtypes = [C.c_char_p, C.POINTER(C.c_ulonglong)]
    stream = torch.cuda.current_stream()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.sharp_b200_kernel_launches()
    lib.sharp_b200_profile(1)
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = lib.sharp_b200_kernel_launches() - launches0
    step_s = ev0.elapsed_time(ev1) * 1e-3 / args.steps
    fam = {}
    for name in ("legendre_synth", "legendre_anal", "ring_synth", "ring_anal", "stage_alm",
                 "scatter_alm"):
        n = C.c_ulonglong(0)
        ms = lib.sharp_b200_profile_ms(name.encode(), C.byref(n))
        fam[name] = (ms, n.value)
    lib.sharp_b200_profile(0)
    if dist:
        tt = torch.tensor([step_s], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        step_s = float(tt.item())
    if args.profile_only:
        if dist:
            dist.destroy_process_group()
        return
    value = world / step_s

    # end-to-end through sharp_execute with pinned host buffers
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    ht, he, hb = (pinned(nalm, torch.complex128) for _ in range(3))
    ht[:], he[:], hb[:] = t, e, b
    hmt, hmq, hmu = (pinned(npix, torch.float64) for _ in range(3))
    hot, hoe, hob = (pinned(nalm, torch.complex128) for _ in range(3))

    def host_step():
        sb.execute(sb.SHARP_ALM2MAP, 0, [ht], [hmt], geom, ainfo, 1, DP)
        sb.execute(sb.SHARP_ALM2MAP, 2, [he, hb], [hmq, hmu], geom, ainfo, 1, DP)
        sb.execute(sb.SHARP_MAP2ALM, 0, [hot], [hmt], geom, ainfo, 1, DP)
        sb.execute(sb.SHARP_MAP2ALM, 2, [hoe, hob], [hmq, hmu], geom, ainfo, 1, DP)

    host_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        host_step()
    e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    if dist:
        tt = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    h2d = 3 * nalm * 16 + 3 * npix * 8
    d2h = 3 * npix * 8 + 3 * nalm * 16

    # correctness of this run's output (round trip without iteration, and
    # GPU-vs-host-API agreement)
    rt_err = float(np.linalg.norm(hot - t) / np.linalg.norm(t))
    api_err = float(np.linalg.norm(ot.cpu().numpy().view(np.complex128) - hot) / np.linalg.norm(hot))

    # roofline of the dominant kernel family (FP64 FMA pipe bound)
    dom = max(("legendre_synth", "legendre_anal"), key=lambda k: fam[k][0])
    dom_ms, dom_n = fam[dom]
    dom_flops = (flops["s0_synth"] + flops["s2_synth"]) if dom == "legendre_synth" else \
        (flops["s0_anal"] + flops["s2_anal"])
    achieved = dom_flops * args.steps / (dom_ms * 1e-3) / 1e12
    peak = fp64_gemm_peak(torch)
    traffic = dram_traffic_from_profiles()
    share = {k: round(v[0] / max(1e-9, sum(x[0] for x in fam.values())), 4) for k, v in fam.items()}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"T+QU alm2map+map2alm, HEALPix Nside {nside}, "
                                   f"lmax=mmax={lmax}, spin 0+2, FP64 drop-in",
                       "nside": nside, "lmax": lmax, "form": "fp64",
                       "alm": "a_lm ~ C_l = (l+1)^-2 exp(-l(l+1) sigma^2), sigma 5', E 0.1, B 0.01",
                       "l2": "inputs larger than L2 (each map 403 MB, each a_lm 134 MB)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp64", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                         "flops_per_launch": dom_flops / 2, "ms_per_launch": dom_ms / max(dom_n, 1),
                         "traffic": traffic},
            "kernel_time_share": share,
            "clocks": clk.summary(),
            "check": {"round_trip_rel_err_no_iteration": rt_err, "device_vs_host_api": api_err}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
