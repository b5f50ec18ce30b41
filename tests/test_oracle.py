"""The oracle is pinned before it is trusted: the numpy restatement must
reproduce the reference test suite's golden values and the reference
library's outputs (committed fixtures and, where built, the library itself)."""
import json
import math
import os

import numpy as np
import pytest

import sht_oracle as so
from helpers import random_alm, rel_l2, uniform_alm

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "sign_scale.json")))
FIX = np.load(os.path.join(HERE, "golden", "reference_small.npz"))


def flipped_gauss():
    geo = so.gauss_geometry(51, 102)
    for r1, r2 in geo.pairs:
        for r in (r1, r2):
            if r is not None:
                r.cth = -r.cth
                r.theta = math.pi - r.theta
    return geo


@pytest.mark.parametrize("key,jtype,spin", [("alm2map_spin0", 1, 0), ("alm2map_spin1", 1, 1),
                                            ("alm2map_spin2", 1, 2), ("alm2map_deriv1", 4, 1)])
def test_oracle_golden_sign_scale(key, jtype, spin):
    geo = flipped_gauss()
    ai = so.triangular_alm_info(50, 50)
    nalm = so.nalm_triangular(50, 50)
    npix = 51 * 102
    na = 1 if (spin == 0 or jtype == 4) else 2
    nm = 1 if (spin == 0 and jtype == 1) else 2
    alms = [np.full(nalm, 1 + 1j) for _ in range(na)]
    maps = [np.zeros(npix) for _ in range(nm)]
    so.execute(jtype, spin, alms, maps, geo, ai, 1, so.SHARP_DP)
    for i, want in enumerate(GOLD[key]):
        got = [maps[i][0], maps[i][npix // 2], maps[i][npix - 1]]
        for j, (g, w) in enumerate(zip(got, want)):
            tol = 1e-11 if (key == "alm2map_deriv1" and i == 0 and j == 0) else 1e-12
            assert abs(g - w) < tol * abs(w), (key, i, j, g, w)


def _fixture_case(name, geo, lmax, mmax, spin, jtype):
    ai = so.triangular_alm_info(lmax, mmax)
    nalm = 1 if (spin == 0 or jtype == 4) else 2
    nmaps = 1 if (spin == 0 and jtype == 1) else 2
    alms = [FIX[f"{name}/alm{i}"] for i in range(nalm)]
    maps = [np.zeros_like(FIX[f"{name}/map{i}"]) for i in range(nmaps)]
    so.execute(jtype, spin, [a.copy() for a in alms], maps, geo, ai, 1, so.SHARP_DP)
    for i in range(nmaps):
        assert rel_l2(maps[i], FIX[f"{name}/map{i}"]) < 1e-13
    if jtype == 1:
        back = [np.zeros_like(alms[0]) for _ in range(nalm)]
        so.execute(0, spin, back, [m.copy() for m in maps], geo, ai, 1, so.SHARP_DP)
        for i in range(nalm):
            assert rel_l2(back[i], FIX[f"{name}/back{i}"]) < 1e-13


def test_oracle_matches_reference_fixtures():
    _fixture_case("hpx16_l32_s0", so.healpix_geometry(16), 32, 32, 0, 1)
    _fixture_case("hpx16_l32_s2", so.healpix_geometry(16), 32, 32, 2, 1)
    _fixture_case("hpx8_l40_m20_s0_alias", so.healpix_geometry(8), 40, 20, 0, 1)
    _fixture_case("gauss_l24_s1_deriv", so.gauss_geometry(25, 50), 24, 24, 1, 4)
    _fixture_case("gauss_l24_s3", so.gauss_geometry(25, 49), 24, 24, 3, 1)


def test_oracle_flags_against_reference_library():
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    nside, lmax = 8, 24
    g = ref.healpix(nside)
    a = ref.triangular(lmax, lmax)
    geo = so.healpix_geometry(nside)
    ai = so.triangular_alm_info(lmax, lmax)
    npix = 12 * nside * nside
    for spin in (0, 2):
        for flags in (16 | 64, 16 | 32):
            na = 1 if spin == 0 else 2
            alms = [uniform_alm(lmax, seed=3 + i, spin=spin) for i in range(na)]
            m_ref = [np.ones(npix) for _ in range(na)]
            m_or = [np.ones(npix) for _ in range(na)]
            ref.execute(1, spin, [x.copy() for x in alms], m_ref, g, a, 1, flags)
            so.execute(1, spin, [x.copy() for x in alms], m_or, geo, ai, 1, flags)
            for i in range(na):
                assert rel_l2(m_or[i], m_ref[i]) < 1e-13
            b_ref = [np.ones_like(alms[0]) for _ in range(na)]
            b_or = [np.ones_like(alms[0]) for _ in range(na)]
            ref.execute(0, spin, b_ref, m_ref, g, a, 1, flags)
            so.execute(0, spin, b_or, [m.copy() for m in m_ref], geo, ai, 1, flags)
            for i in range(na):
                assert rel_l2(b_or[i], b_ref[i]) < 1e-13


def test_oracle_geometry_matches_reference():
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    for nside in (1, 2, 7, 16):
        gobj = ref.healpix(nside)
        g = gobj.ptr.contents
        geo = so.healpix_geometry(nside)
        assert g.npairs == len(geo.pairs)
        # ring indexing (nph, ofs) bit-exact; angles within an ulp or two (the
        # reference is compiled with -ffast-math)
        for i, (r1, r2) in enumerate(geo.pairs):
            p = g.pair[i]
            assert (p.r1.nph, p.r1.ofs) == (r1.nph, r1.ofs)
            assert abs(p.r1.theta - r1.theta) <= 4e-16 * r1.theta
            if r2 is None:
                assert p.r2.nph == -1
            else:
                assert (p.r2.nph, p.r2.ofs) == (r2.nph, r2.ofs)
                assert abs(p.r2.theta - r2.theta) <= 4e-16 * r2.theta


def test_testsuite_lcg_alm():
    # random_alm of sharp_testsuite.c:53-82: values lie in [-1,1), m=0 real
    a = so.testsuite_random_alm(10, 10, 0, 1)
    assert np.all(np.abs(a.real) <= 1) and np.all(a[:11].imag == 0)
    assert len(np.unique(a.real)) > 50


def test_oracle_prime_ring_lengths_against_reference_library():
    # rings whose lengths have large prime factors (61, 127, 97 and twice
    # them, 3 x 37) take the reference's Bluestein and generic-prime FFT
    # paths, and rings shorter than 2 lmax + 1 fold aliased phases; the
    # oracle must agree with the reference library in both directions for
    # spins 0 and 2 on identical rings, angles and weights
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    nph = np.array([61, 127, 122, 254, 111, 64, 97, 194])
    nr = len(nph)
    theta = np.linspace(0.2, math.pi - 0.2, nr)
    ofs = np.concatenate([[0], np.cumsum(nph)[:-1]])
    stride = np.ones(nr, np.int32)
    phi0 = np.linspace(0.0, 0.7, nr)
    wgt = np.linspace(0.5, 1.5, nr) * 4 * math.pi / nph.sum()
    g = ref.general(nph, ofs, stride, phi0, theta, wgt)
    geo = so.make_geom_info(nph, ofs, stride, phi0, theta, wgt)
    lmax = 40
    a = ref.triangular(lmax, lmax)
    ai = so.triangular_alm_info(lmax, lmax)
    npix = int(nph.sum())
    rng = np.random.default_rng(17)
    for spin in (0, 2):
        na = 1 if spin == 0 else 2
        alms = [uniform_alm(lmax, seed=40 + i, spin=spin) for i in range(na)]
        m_ref = [np.zeros(npix) for _ in range(na)]
        m_or = [np.zeros(npix) for _ in range(na)]
        ref.execute(1, spin, [x.copy() for x in alms], m_ref, g, a, 1, 16)
        so.execute(1, spin, [x.copy() for x in alms], m_or, geo, ai, 1, 16)
        for i in range(na):
            assert rel_l2(m_or[i], m_ref[i]) < 1e-12
        maps = [rng.standard_normal(npix) for _ in range(na)]
        b_ref = [np.zeros_like(alms[0]) for _ in range(na)]
        b_or = [np.zeros_like(alms[0]) for _ in range(na)]
        ref.execute(0, spin, b_ref, [m.copy() for m in maps], g, a, 1, 16)
        so.execute(0, spin, b_or, [m.copy() for m in maps], geo, ai, 1, 16)
        for i in range(na):
            assert rel_l2(b_or[i], b_ref[i]) < 1e-12


@pytest.mark.parametrize("spin", [0, 2])
def test_oracle_every_short_ring_length_against_reference_library(spin):
    # rings of every length 1..96 (alias folding for all but the longest at
    # lmax 64, including the one-pixel ring whose m = 1 direct term the
    # reference's fold drops), phi0 shifts and weights, both directions
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    nph = np.arange(1, 97, dtype=np.int32)
    nr = len(nph)
    theta = np.linspace(0.02, np.pi / 2 - 0.02, nr)
    ofs = np.concatenate([[0], np.cumsum(nph)[:-1]])
    st = np.ones(nr, np.int32)
    phi0 = np.linspace(0.0, 1.0, nr)
    w = np.linspace(0.5, 1.5, nr)
    g2 = ref.general(nph, ofs, st, phi0, theta, w)
    go = so.make_geom_info(nph, ofs, st, phi0, theta, w)
    lmax = 64
    a2, ao = ref.triangular(lmax, lmax), so.triangular_alm_info(lmax, lmax)
    na = 1 if spin == 0 else 2
    alms = [uniform_alm(lmax, seed=60 + i, spin=spin) for i in range(na)]
    npix = int(nph.sum())
    m_ref = [np.zeros(npix) for _ in range(na)]
    m_or = [np.zeros(npix) for _ in range(na)]
    ref.execute(1, spin, [x.copy() for x in alms], m_ref, g2, a2, 1, so.SHARP_DP)
    so.execute(so.SHARP_ALM2MAP, spin, [x.copy() for x in alms], m_or, go, ao, 1, so.SHARP_DP)
    for x, y in zip(m_or, m_ref):
        assert rel_l2(x, y) < 1e-13
    rng = np.random.default_rng(5)
    maps = [rng.standard_normal(npix) for _ in range(na)]
    b_ref = [np.zeros_like(alms[0]) for _ in range(na)]
    b_or = [np.zeros_like(alms[0]) for _ in range(na)]
    ref.execute(0, spin, b_ref, [x.copy() for x in maps], g2, a2, 1, so.SHARP_DP)
    so.execute(so.SHARP_MAP2ALM, spin, b_or, [x.copy() for x in maps], go, ao, 1, so.SHARP_DP)
    for x, y in zip(b_or, b_ref):
        assert rel_l2(x, y) < 1e-13
