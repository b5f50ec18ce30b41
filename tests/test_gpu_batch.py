"""sharp_b200_execute_batch: a batch of independent jobs of uneven HEALPix
resolution, lmax and spin (the batched configuration: spin-0 and spin-2
TEB -> IQU sets with Nside drawn from a small set and lmax = 2 Nside, E/B
spectra 0.1 and 0.01 of T), at small sizes and at the configuration's own
size (48 spin-0 + 16 spin-2 sets, Nside 256/512/1024).  Each output must
equal sharp_execute on its own job (FP64) and the reference, and the
SHARP_MIXED batch must stay within 1e-6 relative L2 of FP64 per map."""
import time

import numpy as np
import pytest

import sharp_b200 as sb
from helpers import rel_l2

pytestmark = pytest.mark.gpu
DP, MIXED = sb.SHARP_DP, sb.SHARP_MIXED
TOL_MIXED = 1e-6


def _cl(lmax, fwhm_arcmin=5.0):
    l = np.arange(lmax + 1, dtype=np.float64)
    sig = fwhm_arcmin * np.pi / 10800.0
    cl = np.exp(-l * (l + 1) * sig * sig) / (l + 1) ** 2
    cl[:2] = 0.0
    return cl


def _alm(lmax, cl, rng):
    out = np.zeros(sb.nalm_triangular(lmax), np.complex128)
    i = 0
    for m in range(lmax + 1):
        n = lmax + 1 - m
        a = np.sqrt(cl[m:])
        if m == 0:
            out[i:i + n] = a * rng.standard_normal(n)
        else:
            out[i:i + n] = a * np.sqrt(0.5) * (rng.standard_normal(n)
                                               + 1j * rng.standard_normal(n))
        i += n
    return out


def _mix(nsides=(16, 32, 64), n0=12, n2=4, seed=0):
    """Uneven mix: n0 spin-0 (T) and n2 spin-2 (E, B) sets, Nside uniform over
    nsides, lmax = 2 Nside; one geometry / a_lm object per resolution."""
    rng = np.random.default_rng(seed)
    geo = {n: (sb.Geometry.healpix(n), sb.AlmInfo.triangular(2 * n)) for n in nsides}
    sets = []
    for k in range(n0 + n2):
        spin = 0 if k < n0 else 2
        n = int(rng.choice(nsides))
        cl = _cl(2 * n)
        alms = [_alm(2 * n, cl, rng)] if spin == 0 else \
            [_alm(2 * n, 0.1 * cl, rng), _alm(2 * n, 0.01 * cl, rng)]
        sets.append((spin, n, alms))
    order = rng.permutation(len(sets))   # interleave spins and resolutions
    return geo, [sets[i] for i in order]


def _run_batch(geo, sets, jtype, flags, inputs):
    """One batch call; inputs[i] are the set's input arrays (alm for alm2map,
    maps for map2alm).  Returns the outputs."""
    jobs, outs = [], []
    for (spin, n, _), inp in zip(sets, inputs):
        g, a = geo[n]
        if jtype == sb.SHARP_ALM2MAP:
            out = [np.zeros(12 * n * n) for _ in inp]
            jobs.append((jtype, spin, [x.copy() for x in inp], out, g, a, 1, flags))
        else:
            out = [np.zeros(sb.nalm_triangular(2 * n), np.complex128) for _ in inp]
            jobs.append((jtype, spin, out, [x.copy() for x in inp], g, a, 1, flags))
        outs.append(out)
    ngroups, _ = sb.execute_batch(jobs)
    return ngroups, outs


def _run_single(geo, sets, jtype, flags, inputs):
    outs = []
    for (spin, n, _), inp in zip(sets, inputs):
        g, a = geo[n]
        if jtype == sb.SHARP_ALM2MAP:
            out = [np.zeros(12 * n * n) for _ in inp]
            sb.execute(jtype, spin, [x.copy() for x in inp], out, g, a, 1, flags)
        else:
            out = [np.zeros(sb.nalm_triangular(2 * n), np.complex128) for _ in inp]
            sb.execute(jtype, spin, out, [x.copy() for x in inp], g, a, 1, flags)
        outs.append(out)
    return outs


def test_batch_matches_single_jobs_fp64():
    geo, sets = _mix()
    alms = [s[2] for s in sets]
    ng, maps_b = _run_batch(geo, sets, sb.SHARP_ALM2MAP, DP, alms)
    assert ng == len({(s[0], s[1]) for s in sets})   # one merged job per (spin, Nside)
    maps_s = _run_single(geo, sets, sb.SHARP_ALM2MAP, DP, alms)
    for xb, xs in zip(maps_b, maps_s):
        for x, y in zip(xb, xs):
            assert rel_l2(x, y) < 1e-13
    _, alm_b = _run_batch(geo, sets, sb.SHARP_MAP2ALM, DP, maps_s)
    alm_s = _run_single(geo, sets, sb.SHARP_MAP2ALM, DP, maps_s)
    for xb, xs in zip(alm_b, alm_s):
        for x, y in zip(xb, xs):
            assert rel_l2(x, y) < 1e-13


def test_batch_mixed_error_per_map():
    geo, sets = _mix(seed=1)
    alms = [s[2] for s in sets]
    _, m64 = _run_batch(geo, sets, sb.SHARP_ALM2MAP, DP, alms)
    _, mmx = _run_batch(geo, sets, sb.SHARP_ALM2MAP, DP | MIXED, alms)
    for xb, xs in zip(mmx, m64):
        for x, y in zip(xb, xs):
            assert rel_l2(x, y) < TOL_MIXED
    _, a64 = _run_batch(geo, sets, sb.SHARP_MAP2ALM, DP, m64)
    _, amx = _run_batch(geo, sets, sb.SHARP_MAP2ALM, DP | MIXED, m64)
    for xb, xs in zip(amx, a64):
        for x, y in zip(xb, xs):
            assert rel_l2(x, y) < TOL_MIXED


def test_batch_against_reference():
    import ref
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    geo, sets = _mix(nsides=(16, 32), n0=3, n2=2, seed=2)
    alms = [s[2] for s in sets]
    _, maps_b = _run_batch(geo, sets, sb.SHARP_ALM2MAP, DP, alms)
    rgeo = {n: (ref.healpix(n), ref.triangular(2 * n, 2 * n)) for n in (16, 32)}
    for (spin, n, _), inp, got in zip(sets, alms, maps_b):
        g, a = rgeo[n]
        out = [np.zeros(12 * n * n) for _ in inp]
        ref.execute(sb.SHARP_ALM2MAP, spin, [x.copy() for x in inp], out, g, a, 1, DP)
        for x, y in zip(got, out):
            assert rel_l2(x, y) < 1e-12


def test_batch_device_pointers_and_merge_limit():
    import torch
    dev = torch.device("cuda:0")
    nside, lmax = 16, 32
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    rng = np.random.default_rng(3)
    nalm = sb.nalm_triangular(lmax)
    # 60 + 60 single-transform jobs: merged into two jobs (at most 100 each)
    alms = [rng.standard_normal(nalm) + 1j * rng.standard_normal(nalm) for _ in range(120)]
    for x in alms:
        x[:lmax + 1] = x[:lmax + 1].real
    ta = [torch.view_as_real(torch.from_numpy(x).to(dev)).reshape(-1) for x in alms]
    tm = [torch.zeros(12 * nside * nside, dtype=torch.float64, device=dev) for _ in alms]
    jobs = [(sb.SHARP_ALM2MAP, 0, [ta[i]], [tm[i]], g, a, 1, DP) for i in range(120)]
    ng, op = sb.execute_batch(jobs, device=True)
    torch.cuda.synchronize()
    assert ng == 2 and op > 0
    for i in (0, 57, 119):
        ref_map = [np.zeros(12 * nside * nside)]
        sb.execute(sb.SHARP_ALM2MAP, 0, [alms[i].copy()], ref_map, g, a, 1, DP)
        assert rel_l2(tm[i].cpu().numpy(), ref_map[0]) < 1e-13


def test_config2_full_size_per_map_errors():
    # the batched configuration at its stated size: 48 spin-0 + 16 spin-2
    # sets, Nside uniform over {256, 512, 1024}, lmax = 2 Nside, one batch
    # call per direction and precision.  FP64 against the reference on a
    # subset of sets (1e-12); SHARP_MIXED against FP64 on every map (1e-6),
    # the per-map errors printed.
    import ref
    geo, sets = _mix(nsides=(256, 512, 1024), n0=48, n2=16, seed=5)
    alms = [s[2] for s in sets]
    t0 = time.perf_counter()
    _, m64 = _run_batch(geo, sets, sb.SHARP_ALM2MAP, DP, alms)
    t1 = time.perf_counter()
    _, mmx = _run_batch(geo, sets, sb.SHARP_ALM2MAP, DP | MIXED, alms)
    t2 = time.perf_counter()
    _, a64 = _run_batch(geo, sets, sb.SHARP_MAP2ALM, DP, m64)
    _, amx = _run_batch(geo, sets, sb.SHARP_MAP2ALM, DP | MIXED, m64)
    emap = [rel_l2(x, y) for xb, yb in zip(mmx, m64) for x, y in zip(xb, yb)]
    ealm = [rel_l2(x, y) for xb, yb in zip(amx, a64) for x, y in zip(xb, yb)]
    print(f"config 2: {len(sets)} sets, {len(emap)} maps; host-array batch alm2map "
          f"FP64 {t1 - t0:.2f} s, mixed {t2 - t1:.2f} s; mixed vs FP64 per map: "
          f"maps max {max(emap):.2e} median {np.median(emap):.2e}, "
          f"a_lm max {max(ealm):.2e} median {np.median(ealm):.2e}")
    assert max(emap) < TOL_MIXED and max(ealm) < TOL_MIXED
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    # reference on one spin-0 and one spin-2 set of each resolution
    pick = {}
    for i, (spin, n, _) in enumerate(sets):
        pick.setdefault((spin, n), i)
    for (spin, n), i in sorted(pick.items()):
        g, a = ref.healpix(n), ref.triangular(2 * n, 2 * n)
        out = [np.zeros(12 * n * n) for _ in alms[i]]
        ref.execute(sb.SHARP_ALM2MAP, spin, [x.copy() for x in alms[i]], out, g, a, 1, DP)
        for x, y in zip(m64[i], out):
            assert rel_l2(x, y) < 1e-12
        back = [np.zeros_like(x) for x in alms[i]]
        ref.execute(sb.SHARP_MAP2ALM, spin, back, [x.copy() for x in m64[i]], g, a, 1, DP)
        for x, y in zip(a64[i], back):
            assert rel_l2(x, y) < 1e-12


def test_config2_device_batch_runs_groups_side_by_side():
    # the batched configuration with device arrays: one batch call runs its
    # six merged groups (spin x Nside) side by side on library streams; the
    # outputs equal those of the same groups run one after another, bit for
    # bit, and the two times are printed
    import torch
    geo, sets = _mix(nsides=(256, 512, 1024), n0=48, n2=16, seed=6)
    dev = torch.device("cuda:0")

    def dalm(x):
        return torch.view_as_real(torch.from_numpy(x).to(dev)).reshape(-1)

    alms = [[dalm(x) for x in s[2]] for s in sets]
    out_b = [[torch.zeros(12 * s[1] ** 2, dtype=torch.float64, device=dev) for _ in s[2]]
             for s in sets]
    out_s = [[torch.zeros_like(x) for x in o] for o in out_b]
    for flags in (DP, DP | MIXED):
        jobs_b = [(sb.SHARP_ALM2MAP, s[0], a, o, *geo[s[1]], 1, flags)
                  for s, a, o in zip(sets, alms, out_b)]
        sb.execute_batch(jobs_b, device=True)          # warm-up: plans, tables
        # the same merged groups, one after another on the current stream
        groups = {}
        for s, a, o in zip(sets, alms, out_s):
            g = groups.setdefault((s[0], s[1]), ([], []))
            g[0].extend(a)
            g[1].extend(o)
        def sequential():
            for (spin, n), (a, o) in groups.items():
                nt = len(a) // (1 if spin == 0 else 2)
                sb.execute_device(sb.SHARP_ALM2MAP, spin, a, o, *geo[n], nt, flags)
        sequential()
        torch.cuda.synchronize()
        times = {}
        for name, fn in (("batch", lambda: sb.execute_batch(jobs_b, device=True)),
                         ("sequential", sequential)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            times[name] = e0.elapsed_time(e1)
        print(f"config 2 alm2map, {'mixed' if flags & MIXED else 'FP64'}: batch "
              f"{times['batch']:.1f} ms, groups one after another {times['sequential']:.1f} ms")
        for xb, xs in zip(out_b, out_s):
            for x, y in zip(xb, xs):
                assert torch.equal(x, y)


def test_host_batch_round_trip_in_one_call():
    # alm2map jobs and the map2alm jobs of their maps in one host-array call:
    # the map2alm input copies must wait for the alm2map output copies (the
    # maps start as zeros).  The maps are slices of one buffer (each its own
    # base pointer), several pieces per job, spin 0 and 2; a third job
    # compatible with the first comes after the dependent ones and must not
    # be merged ahead of them.  Every output equals the sequential calls.
    nside, lmax, nt = 32, 64, 7
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    npix, nalm = 12 * nside * nside, sb.nalm_triangular(lmax)
    rng = np.random.default_rng(11)
    cl = _cl(lmax)
    alm0 = [_alm(lmax, cl, rng) for _ in range(nt)]
    alm2 = [_alm(lmax, 0.1 * cl, rng) for _ in range(2 * nt)]
    big = np.zeros(3 * nt * npix)
    m0 = [big[i * npix:(i + 1) * npix] for i in range(nt)]
    m2 = [big[(nt + i) * npix:(nt + i + 1) * npix] for i in range(2 * nt)]
    o0 = [np.zeros(nalm, np.complex128) for _ in range(nt)]
    o2 = [np.zeros(nalm, np.complex128) for _ in range(2 * nt)]
    extra = [np.zeros(npix) for _ in range(2)]
    jobs = [(sb.SHARP_ALM2MAP, 0, alm0, m0, g, a, nt, DP),
            (sb.SHARP_ALM2MAP, 2, alm2, m2, g, a, nt, DP),
            (sb.SHARP_MAP2ALM, 0, o0, m0, g, a, nt, DP),
            (sb.SHARP_MAP2ALM, 2, o2, m2, g, a, nt, DP),
            (sb.SHARP_ALM2MAP, 0, alm0[:2], extra, g, a, 2, DP)]
    ng, _ = sb.execute_batch(jobs)
    assert ng == 5
    r0 = [np.zeros(npix) for _ in range(nt)]
    r2 = [np.zeros(npix) for _ in range(2 * nt)]
    sb.execute(sb.SHARP_ALM2MAP, 0, [x.copy() for x in alm0], r0, g, a, nt, DP)
    sb.execute(sb.SHARP_ALM2MAP, 2, [x.copy() for x in alm2], r2, g, a, nt, DP)
    q0 = [np.zeros(nalm, np.complex128) for _ in range(nt)]
    q2 = [np.zeros(nalm, np.complex128) for _ in range(2 * nt)]
    sb.execute(sb.SHARP_MAP2ALM, 0, q0, [x.copy() for x in r0], g, a, nt, DP)
    sb.execute(sb.SHARP_MAP2ALM, 2, q2, [x.copy() for x in r2], g, a, nt, DP)
    for got, want in zip(m0 + m2 + o0 + o2, r0 + r2 + q0 + q2):
        assert np.array_equal(got, want)
    for got, want in zip(extra, r0[:2]):
        assert rel_l2(got, want) < 1e-13
    # independent jobs still merge across the list
    outs = [np.zeros(npix) for _ in range(3)]
    ng, _ = sb.execute_batch([(sb.SHARP_ALM2MAP, 0, [alm0[0]], [outs[0]], g, a, 1, DP),
                              (sb.SHARP_MAP2ALM, 0, [q0[0].copy()], [r0[1].copy()], g, a, 1, DP),
                              (sb.SHARP_ALM2MAP, 0, [alm0[2]], [outs[2]], g, a, 1, DP)])
    assert ng == 2
    assert rel_l2(outs[0], r0[0]) < 1e-13 and rel_l2(outs[2], r0[2]) < 1e-13
