"""sharp_b200_batch_groups (host only): how a batch is merged.  Host-array
batches whose jobs read what another job writes (byte ranges of the arrays,
so slices of one buffer count) merge only consecutive jobs; independent
batches, and device-pointer batches, merge compatible jobs anywhere in the
list, up to 100 transforms per group."""
import numpy as np
import torch

import sharp_b200 as sb

DP = sb.SHARP_DP


def _setup(nside=8, lmax=16):
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    return g, a, 12 * nside * nside, sb.nalm_triangular(lmax)


def test_independent_jobs_merge_across_the_list():
    g1, a1, npix1, nalm1 = _setup(8, 16)
    g2, a2, npix2, nalm2 = _setup(16, 32)
    jobs = []
    for k in range(4):
        g, a, npix, nalm = (g1, a1, npix1, nalm1) if k % 2 == 0 else (g2, a2, npix2, nalm2)
        jobs.append((sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], [np.zeros(npix)],
                     g, a, 1, DP))
    assert sb.batch_groups(jobs) == [0, 1, 0, 1]


def test_round_trip_merges_only_consecutive_jobs():
    g, a, npix, nalm = _setup()
    maps = [np.zeros(npix)]
    jobs = [(sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], maps, g, a, 1, DP),
            (sb.SHARP_MAP2ALM, 0, [np.zeros(nalm, np.complex128)], maps, g, a, 1, DP),
            (sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], [np.zeros(npix)], g, a, 1, DP),
            (sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], [np.zeros(npix)], g, a, 1, DP)]
    # the third job may not move ahead of the map2alm; the fourth joins the third
    assert sb.batch_groups(jobs) == [0, 1, 2, 2]


def test_overlap_is_found_through_slices_and_write_after_read():
    g, a, npix, nalm = _setup()
    big = np.zeros(3 * npix)
    out = big[:npix]
    shifted = big[npix // 2:npix // 2 + npix]    # another base pointer, overlapping bytes
    jobs = [(sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], [out], g, a, 1, DP),
            (sb.SHARP_MAP2ALM, 0, [np.zeros(nalm, np.complex128)], [shifted], g, a, 1, DP),
            (sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], [big[2 * npix:]], g, a, 1, DP)]
    assert sb.batch_groups(jobs) == [0, 1, 2]
    # disjoint slices of the same buffer are independent
    jobs[1] = (sb.SHARP_MAP2ALM, 0, [np.zeros(nalm, np.complex128)], [big[npix:2 * npix]],
               g, a, 1, DP)
    assert sb.batch_groups(jobs) == [0, 1, 0]
    # a map2alm that reads a map a later alm2map overwrites
    m = [np.zeros(npix)]
    jobs = [(sb.SHARP_MAP2ALM, 0, [np.zeros(nalm, np.complex128)], m, g, a, 1, DP),
            (sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], [np.zeros(npix)], g, a, 1, DP),
            (sb.SHARP_MAP2ALM, 0, [np.zeros(nalm, np.complex128)], [np.zeros(npix)], g, a, 1, DP),
            (sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], m, g, a, 1, DP)]
    assert sb.batch_groups(jobs) == [0, 1, 2, 3]


def test_spin_jobs_and_device_pointers():
    g, a, npix, nalm = _setup()
    m = [np.zeros(npix), np.zeros(npix)]
    jobs = [(sb.SHARP_ALM2MAP, 2, [np.zeros(nalm, np.complex128) for _ in range(2)], m,
             g, a, 1, DP),
            (sb.SHARP_MAP2ALM, 2, [np.zeros(nalm, np.complex128) for _ in range(2)], m,
             g, a, 1, DP),
            (sb.SHARP_ALM2MAP, 2, [np.zeros(nalm, np.complex128) for _ in range(2)],
             [np.zeros(npix), np.zeros(npix)], g, a, 1, DP)]
    assert sb.batch_groups(jobs) == [0, 1, 2]
    # device pointers: the jobs are independent by contract, so merging is free
    t = [torch.zeros(npix, dtype=torch.float64) for _ in range(4)]
    ta = [torch.zeros(2 * nalm, dtype=torch.float64) for _ in range(6)]
    jobs = [(sb.SHARP_ALM2MAP, 2, ta[0:2], t[0:2], g, a, 1, DP),
            (sb.SHARP_MAP2ALM, 2, ta[2:4], t[0:2], g, a, 1, DP),
            (sb.SHARP_ALM2MAP, 2, ta[4:6], t[2:4], g, a, 1, DP)]
    assert sb.batch_groups(jobs, device=True) == [0, 1, 0]


def test_merge_limit_of_100_transforms():
    g, a, npix, nalm = _setup()
    jobs = [(sb.SHARP_ALM2MAP, 0, [np.zeros(nalm, np.complex128)], [np.zeros(npix)], g, a, 1, DP)
            for _ in range(120)]
    of = sb.batch_groups(jobs)
    assert of[:100] == [0] * 100 and of[100:] == [1] * 20
