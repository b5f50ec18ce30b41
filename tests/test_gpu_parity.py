"""GPU parity: the CUDA engine, called through the C ABI, against the
reference libsharp (oracle/_ref) and the committed golden values.

Tolerances: FP64 paths within 1e-12 relative L2 of the reference;
single-precision I/O within 1e-6; the reference test
suite's own known answers at its own tolerances (1e-12 / 1e-11)."""
import json
import math
import os

import numpy as np
import pytest

import sharp_b200 as sb
import sht_oracle as so
from helpers import random_alm, rel_l2, uniform_alm, cl_spectrum

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "sign_scale.json")))
FIX = np.load(os.path.join(HERE, "golden", "reference_small.npz"))
DP = sb.SHARP_DP
TOL = 1e-12


@pytest.fixture(scope="module")
def ref():
    import ref as r
    if not r.available():
        pytest.skip("reference library not built (make -C oracle)")
    return r


def _nmaps(jtype, spin):
    return 1 if (spin == 0 and jtype != 4) else 2


def _nalm(jtype, spin):
    return 1 if (spin == 0 or jtype == 4) else 2


def run_pair(ref, gspec, lmax, mmax, spin, jtype, flags=DP, ntrans=1, seed=0, out_init=0.0):
    """Runs the same job on the GPU engine and the reference, returns both outputs."""
    if gspec[0] == "healpix":
        g_ours, g_ref = sb.Geometry.healpix(gspec[1]), ref.healpix(gspec[1])
    else:
        g_ours, g_ref = sb.Geometry.grid(*gspec), ref.grid(*gspec)
    a_ours, a_ref = sb.AlmInfo.triangular(lmax, mmax), ref.triangular(lmax, mmax)
    npix = g_ref.npix()
    na, nm = _nalm(jtype, spin) * ntrans, _nmaps(jtype, spin) * ntrans
    ncpx = np.complex128 if flags & DP else np.complex64
    nreal = np.float64 if flags & DP else np.float32
    nalm = sb.nalm_triangular(lmax, mmax)
    rng = np.random.default_rng(seed)
    if jtype in (0, 2):  # analysis types take maps
        maps = [rng.standard_normal(npix).astype(nreal) for _ in range(nm)]
        o1 = [np.full(nalm, out_init, ncpx) for _ in range(na)]
        o2 = [x.copy() for x in o1]
        sb.execute(jtype, spin, o1, [m.copy() for m in maps], g_ours, a_ours, ntrans, flags)
        ref.execute(jtype, spin, o2, [m.copy() for m in maps], g_ref, a_ref, ntrans, flags)
    else:
        alms = [uniform_alm(lmax, mmax, seed=seed + i, spin=spin).astype(ncpx) for i in range(na)]
        o1 = [np.full(npix, out_init, nreal) for _ in range(nm)]
        o2 = [x.copy() for x in o1]
        sb.execute(jtype, spin, [a.copy() for a in alms], o1, g_ours, a_ours, ntrans, flags)
        ref.execute(jtype, spin, [a.copy() for a in alms], o2, g_ref, a_ref, ntrans, flags)
    return o1, o2


def test_golden_sign_scale_on_gpu():
    # libsharp/sharp_testsuite.c:337-443, ntrans 1..9 as there
    g = sb.Geometry.grid("gauss", 51, 102)
    gi = g.ptr.contents
    for i in range(gi.npairs):
        for r in (gi.pair[i].r1, gi.pair[i].r2):
            r.cth = -r.cth
            r.theta = math.pi - r.theta
    a = sb.AlmInfo.triangular(50, 50)
    npix, nalm = 51 * 102, sb.nalm_triangular(50)
    for ntrans in (1, 2, 3, 5, 9):
        for key, jt, spin in (("alm2map_spin0", 1, 0), ("alm2map_spin1", 1, 1),
                              ("alm2map_spin2", 1, 2), ("alm2map_deriv1", 4, 1)):
            na, nm = _nalm(jt, spin), _nmaps(jt, spin)
            alms = [np.full(nalm, 1 + 1j) for _ in range(na * ntrans)]
            maps = [np.zeros(npix) for _ in range(nm * ntrans)]
            sb.execute(jt, spin, alms, maps, g, a, ntrans, DP)
            for it in range(ntrans):
                for i, want in enumerate(GOLD[key]):
                    mp = maps[it * nm + i]
                    got = [mp[0], mp[npix // 2], mp[npix - 1]]
                    for j, (gv, w) in enumerate(zip(got, want)):
                        tol = 1e-11 if (key == "alm2map_deriv1" and i == 0 and j == 0) else 1e-12
                        assert abs(gv - w) < tol * abs(w), (ntrans, key, i, j, gv, w)


@pytest.mark.parametrize("name,geo,lmax,mmax,spin,jtype", [
    ("hpx16_l32_s0", ("healpix", 16), 32, 32, 0, 1),
    ("hpx16_l32_s2", ("healpix", 16), 32, 32, 2, 1),
    ("hpx8_l40_m20_s0_alias", ("healpix", 8), 40, 20, 0, 1),
    ("gauss_l24_s1_deriv", ("gauss", 25, 50), 24, 24, 1, 4),
    ("gauss_l24_s3", ("gauss", 25, 49), 24, 24, 3, 1)])
def test_committed_reference_fixtures(name, geo, lmax, mmax, spin, jtype):
    g = sb.Geometry.healpix(geo[1]) if geo[0] == "healpix" else sb.Geometry.grid(*geo)
    a = sb.AlmInfo.triangular(lmax, mmax)
    na, nm = _nalm(jtype, spin), _nmaps(jtype, spin)
    alms = [FIX[f"{name}/alm{i}"].copy() for i in range(na)]
    maps = [np.zeros_like(FIX[f"{name}/map{i}"]) for i in range(nm)]
    sb.execute(jtype, spin, alms, maps, g, a, 1, DP)
    for i in range(nm):
        assert rel_l2(maps[i], FIX[f"{name}/map{i}"]) < TOL
    if jtype == 1:
        back = [np.zeros_like(alms[0]) for _ in range(na)]
        sb.execute(0, spin, back, maps, g, a, 1, DP)
        for i in range(na):
            assert rel_l2(back[i], FIX[f"{name}/back{i}"]) < TOL


def test_config0_nside64_lmax128_both_directions(ref):
    for jt in (1, 0):
        o1, o2 = run_pair(ref, ("healpix", 64), 128, 128, 0, jt)
        assert rel_l2(o1[0], o2[0]) < TOL


def test_config0_against_numpy_oracle():
    nside, lmax = 64, 128
    g = sb.Geometry.healpix(nside)
    a = sb.AlmInfo.triangular(lmax)
    alm = random_alm(lmax, seed=0)
    mp = np.zeros(12 * nside * nside)
    sb.execute(1, 0, [alm.copy()], [mp], g, a, 1, DP)
    mo = np.zeros_like(mp)
    so.execute(1, 0, [alm.copy()], [mo], so.healpix_geometry(nside), so.triangular_alm_info(lmax, lmax), 1, DP)
    assert rel_l2(mp, mo) < TOL
    b1 = np.zeros_like(alm); b2 = np.zeros_like(alm)
    sb.execute(0, 0, [b1], [mp.copy()], g, a, 1, DP)
    so.execute(0, 0, [b2], [mp.copy()], so.healpix_geometry(nside), so.triangular_alm_info(lmax, lmax), 1, DP)
    assert rel_l2(b1, b2) < TOL


@pytest.mark.parametrize("spin", [0, 1, 2, 3, 30])
def test_acctest_gauss_round_trip(spin):
    # libsharp/sharp_testsuite.c:490-529: Gauss lmax=mmax=127, 128x256, ntrans 1..6
    g = sb.Geometry.grid("gauss", 128, 256)
    a = sb.AlmInfo.triangular(127)
    nalm = sb.nalm_triangular(127)
    for ntrans in range(1, 7):
        na = _nalm(1, spin) * ntrans
        alms = [uniform_alm(127, seed=17 * ntrans + i, spin=spin) for i in range(na)]
        maps = [np.zeros(128 * 256) for _ in range(_nmaps(1, spin) * ntrans)]
        sb.execute(1, spin, [x.copy() for x in alms], maps, g, a, ntrans, DP)
        back = [np.zeros(nalm, np.complex128) for _ in range(na)]
        sb.execute(0, spin, back, maps, g, a, ntrans, DP)
        for x, y in zip(alms, back):
            err = y - x
            assert np.sqrt(np.mean(np.abs(err) ** 2) / np.mean(np.abs(x) ** 2)) < 1e-10
            assert np.abs(err).max() < 1e-10


@pytest.mark.parametrize("spin", [0, 2])
@pytest.mark.parametrize("jtype", [1, 0, 2, 3])
@pytest.mark.parametrize("flags", [DP, DP | sb.SHARP_ADD, DP | sb.SHARP_REAL_HARMONICS])
def test_types_and_flags_match_reference(ref, spin, jtype, flags):
    o1, o2 = run_pair(ref, ("healpix", 16), 40, 40, spin, jtype, flags, ntrans=2, out_init=0.25)
    for x, y in zip(o1, o2):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spin,jtype", [(0, 1), (0, 0), (2, 1), (2, 0)])
def test_single_precision_io_matches_reference(ref, spin, jtype):
    o1, o2 = run_pair(ref, ("healpix", 16), 32, 32, spin, jtype, flags=0)
    for x, y in zip(o1, o2):
        assert x.dtype in (np.float32, np.complex64)
        assert rel_l2(x, y) < 1e-6


@pytest.mark.parametrize("ntrans", [1, 3, 5])
def test_deriv1_and_ntrans_match_reference(ref, ntrans):
    o1, o2 = run_pair(ref, ("healpix", 16), 48, 48, 1, 4, ntrans=ntrans)
    for x, y in zip(o1, o2):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spin", [0, 1, 2, 5])
def test_alias_and_partial_mmax_match_reference(ref, spin):
    for gspec, lmax, mmax in ((("healpix", 8), 40, 20), (("healpix", 4), 30, 30),
                              (("fejer1", 31, 30), 30, 14), (("cc", 33, 33), 24, 24),
                              (("mw", 30, 59), 29, 29), (("fejer2", 31, 61), 30, 30)):
        for jt in (1, 0):
            if jt == 0 and gspec[0] == "mw":
                continue
            o1, o2 = run_pair(ref, gspec, lmax, mmax, spin, jt)
            for x, y in zip(o1, o2):
                assert rel_l2(x, y) < TOL, (gspec, lmax, mmax, spin, jt)


@pytest.mark.parametrize("spin", [0, 1, 2, 4])
def test_conviqt_style_odd_rings_match_reference(ref, spin):
    # conviqt_v4_module.cc:160-181: equidistant theta, nph = 2*olmax+1, phi0 = pi/2,
    # no weights, alm2map (k=0) / alm2map_spin (k>0)
    olmax = 37
    nr = olmax + 1
    theta = (np.arange(nr) + 0.5) * np.pi / nr
    nph = np.full(nr, 2 * olmax + 1, np.int32)
    ofs = np.arange(nr) * (2 * olmax + 1)
    st = np.ones(nr, np.int32)
    phi0 = np.full(nr, np.pi / 2)
    g1 = sb.Geometry.general(nph, ofs, st, phi0, theta)
    g2 = ref.general(nph, ofs, st, phi0, theta)
    a1, a2 = sb.AlmInfo.triangular(olmax), ref.triangular(olmax, olmax)
    na = _nalm(1, spin)
    alms = [uniform_alm(olmax, seed=9 + i, spin=spin) for i in range(na)]
    m1 = [np.zeros(nr * (2 * olmax + 1)) for _ in range(na)]
    m2 = [np.zeros_like(x) for x in m1]
    sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, DP)
    ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, DP)
    for x, y in zip(m1, m2):
        assert rel_l2(x, y) < TOL


def test_no_fft_matches_reference(ref):
    lmax = 20
    nr = 22
    theta = (np.arange(nr) + 0.5) * np.pi / nr
    nph = np.full(nr, lmax + 1, np.int32)
    ofs = np.arange(nr) * (lmax + 1)
    st = np.ones(nr, np.int32)
    w = np.linspace(0.5, 1.0, nr)
    g1 = sb.Geometry.general(nph, ofs, st, np.zeros(nr), theta, w)
    g2 = ref.general(nph, ofs, st, np.zeros(nr), theta, w)
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    for spin in (0, 2):
        na = _nalm(1, spin)
        alms = [uniform_alm(lmax, seed=4 + i, spin=spin) for i in range(na)]
        f = DP | sb.SHARP_NO_FFT
        m1 = [np.zeros(nr * (lmax + 1), np.complex128) for _ in range(na)]
        m2 = [np.zeros_like(x) for x in m1]
        sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, f)
        ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, f)
        for x, y in zip(m1, m2):
            assert rel_l2(x, y) < TOL
        b1 = [np.zeros_like(alms[0]) for _ in range(na)]
        b2 = [np.zeros_like(alms[0]) for _ in range(na)]
        sb.execute(0, spin, b1, [x.copy() for x in m2], g1, a1, 1, f)
        ref.execute(0, spin, b2, [x.copy() for x in m2], g2, a2, 1, f)
        for x, y in zip(b1, b2):
            assert rel_l2(x, y) < TOL


def test_packed_and_rectangular_alm_layouts(ref):
    nside, lmax = 8, 16
    g1, g2 = sb.Geometry.healpix(nside), ref.healpix(nside)
    npix = 12 * nside * nside
    # rectangular (Fortran Healpix) layout with holes for l<m
    r1 = sb.AlmInfo.rectangular(lmax)
    rng = np.random.default_rng(1)
    alm = rng.standard_normal((lmax + 1) ** 2) + 1j * rng.standard_normal((lmax + 1) ** 2)
    alm[: lmax + 1] = alm[: lmax + 1].real
    from ref import AlmInfo as _A  # noqa: F401
    mv = np.arange(lmax + 1)
    r2 = ref.general_alm(lmax, mv, mv * (lmax + 1))
    m1, m2 = np.zeros(npix), np.zeros(npix)
    sb.execute(1, 0, [alm.copy()], [m1], g1, r1, 1, DP)
    ref.execute(1, 0, [alm.copy()], [m2], g2, r2, 1, DP)
    assert rel_l2(m1, m2) < TOL
    b1 = np.full_like(alm, 7.0); b2 = np.full_like(alm, 7.0)
    sb.execute(0, 0, [b1], [m2.copy()], g1, r1, 1, DP)
    ref.execute(0, 0, [b2], [m2.copy()], g2, r2, 1, DP)
    assert rel_l2(b1, b2) < TOL  # holes (l<m) keep their 7.0
    # SHARP_PACKED: m=0 stored as reals, mvstart in reals
    starts = [0]
    for m in range(1, lmax + 1):
        prev = starts[-1] + ((lmax + 1) if m == 1 else 2 * (lmax - m + 2))
        starts.append(prev)
    mvs = np.array([0] + [starts[m] - 2 * m for m in range(1, lmax + 1)])
    total = (lmax + 1) + 2 * sum(lmax - m + 1 for m in range(1, lmax + 1))
    flat = rng.standard_normal(total)
    p1 = sb.AlmInfo.general(lmax, mv, mvs, 1, sb.SHARP_PACKED)
    p2 = ref.general_alm(lmax, mv, mvs, 1, 1)
    m1, m2 = np.zeros(npix), np.zeros(npix)
    sb.execute(1, 0, [flat.copy()], [m1], g1, p1, 1, DP)
    ref.execute(1, 0, [flat.copy()], [m2], g2, p2, 1, DP)
    assert rel_l2(m1, m2) < TOL
    f1 = np.zeros(total); f2 = np.zeros(total)
    sb.execute(0, 0, [f1], [m2.copy()], g1, p1, 1, DP)
    ref.execute(0, 0, [f2], [m2.copy()], g2, p2, 1, DP)
    assert rel_l2(f1, f2) < TOL


def test_adjoint_flag_is_transpose(ref):
    # <Y a, x> = sum_{m=0} Re(a* Yt x) + 2 sum_{m>0} Re(a* Yt x)
    nside, lmax = 16, 40
    g = sb.Geometry.healpix(nside)
    a = sb.AlmInfo.triangular(lmax)
    rng = np.random.default_rng(3)
    for spin in (0, 2):
        na = _nalm(1, spin)
        alms = [uniform_alm(lmax, seed=20 + i, spin=spin) for i in range(na)]
        x = [rng.standard_normal(12 * nside * nside) for _ in range(na)]
        ya = [np.zeros_like(x[0]) for _ in range(na)]
        sb.execute(1, spin, [v.copy() for v in alms], ya, g, a, 1, DP)
        ytx = [np.zeros_like(alms[0]) for _ in range(na)]
        sb.execute(1, spin, ytx, [v.copy() for v in x], g, a, 1, DP | sb.SHARP_ADJOINT)
        lhs = sum(np.dot(u, v) for u, v in zip(ya, x))
        wts = np.full(len(alms[0]), 2.0)
        wts[: lmax + 1] = 1.0  # m = 0 block of the triangular layout
        rhs = sum(np.sum(wts * (np.conj(u) * v).real) for u, v in zip(alms, ytx))
        assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def _iterate_map2alm(execute, g, a, mp, nalm, niter):
    # map2alm_iter, Healpix_cxx/alm_healpix_tools.cc:73-85
    alm = np.zeros(nalm, np.complex128)
    execute(0, 0, [alm], [mp.copy()], g, a, 1, DP)
    for _ in range(niter):
        m2 = np.zeros_like(mp)
        execute(1, 0, [alm.copy()], [m2], g, a, 1, DP)
        execute(0, 0, [alm], [mp - m2], g, a, 1, DP | sb.SHARP_ADD)
    return alm


def test_config1_nside1024_lmax2048_with_jacobi_iterations(ref):
    nside, lmax = 1024, 2048
    g1, g2 = sb.Geometry.healpix(nside), ref.healpix(nside)
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    alm = random_alm(lmax, seed=0, cl=cl_spectrum(lmax, beam_arcmin=5.0))
    m1 = np.zeros(12 * nside * nside); m2 = np.zeros_like(m1)
    sb.execute(1, 0, [alm.copy()], [m1], g1, a1, 1, DP)
    ref.execute(1, 0, [alm.copy()], [m2], g2, a2, 1, DP)
    assert rel_l2(m1, m2) < TOL
    b1 = _iterate_map2alm(sb.execute, g1, a1, m2, len(alm), 3)
    b2 = _iterate_map2alm(ref.execute, g2, a2, m2, len(alm), 3)
    assert rel_l2(b1, b2) < TOL
    # the Jacobi sweeps move the estimate towards the input a_lm
    b0 = _iterate_map2alm(sb.execute, g1, a1, m2, len(alm), 0)
    assert rel_l2(b1, alm) < rel_l2(b0, alm)


def test_metric_config_nside2048_lmax4096_spin0_and_spin2(ref):
    nside, lmax = 2048, 4096
    g1, g2 = sb.Geometry.healpix(nside), ref.healpix(nside)
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    cl = cl_spectrum(lmax, beam_arcmin=5.0)
    rng = np.random.default_rng(7)
    t = random_alm(lmax, cl=cl, rng=rng)
    e = random_alm(lmax, cl=0.1 * cl, rng=rng)
    b = random_alm(lmax, cl=0.01 * cl, rng=rng)
    npix = 12 * nside * nside
    m1, m2 = np.zeros(npix), np.zeros(npix)
    sb.execute(1, 0, [t.copy()], [m1], g1, a1, 1, DP)
    ref.execute(1, 0, [t.copy()], [m2], g2, a2, 1, DP)
    assert rel_l2(m1, m2) < TOL
    q1, u1, q2, u2 = (np.zeros(npix) for _ in range(4))
    sb.execute(1, 2, [e.copy(), b.copy()], [q1, u1], g1, a1, 1, DP)
    ref.execute(1, 2, [e.copy(), b.copy()], [q2, u2], g2, a2, 1, DP)
    assert rel_l2(q1, q2) < TOL and rel_l2(u1, u2) < TOL
    x1 = [np.zeros_like(e), np.zeros_like(e)]
    x2 = [np.zeros_like(e), np.zeros_like(e)]
    sb.execute(0, 2, x1, [q2.copy(), u2.copy()], g1, a1, 1, DP)
    ref.execute(0, 2, x2, [q2.copy(), u2.copy()], g2, a2, 1, DP)
    assert rel_l2(x1[0], x2[0]) < TOL and rel_l2(x1[1], x2[1]) < TOL
    # spin-0 analysis of the reference's T map
    y1, y2 = np.zeros_like(t), np.zeros_like(t)
    sb.execute(0, 0, [y1], [m2.copy()], g1, a1, 1, DP)
    ref.execute(0, 0, [y2], [m2.copy()], g2, a2, 1, DP)
    assert rel_l2(y1, y2) < TOL


def test_config4_nside4096_lmax8192_fp64_matches_reference(ref):
    # the large polarised configuration in FP64 against the reference:
    # Nside 4096 (rings up to 16384 pixels), lmax = mmax = 8192, spin 0 and 2,
    # both directions, with its spectra (C_l^T with a 1-arcmin beam, E and B
    # at 0.1 and 0.01 of it).  This pins the scaled run-up of the recurrence
    # for m up to 8192 on the reference itself (libsharp/sharp_core_inc.c).
    nside, lmax = 4096, 8192
    g1, g2 = sb.Geometry.healpix(nside), ref.healpix(nside)
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    cl = cl_spectrum(lmax, beam_arcmin=1.0)
    rng = np.random.default_rng(41)
    npix = 12 * nside * nside
    t = random_alm(lmax, cl=cl, rng=rng)
    m1, m2 = np.zeros(npix), np.zeros(npix)
    sb.execute(1, 0, [t.copy()], [m1], g1, a1, 1, DP)
    ref.execute(1, 0, [t.copy()], [m2], g2, a2, 1, DP)
    assert rel_l2(m1, m2) < TOL
    y1, y2 = np.zeros_like(t), np.zeros_like(t)
    sb.execute(0, 0, [y1], [m2], g1, a1, 1, DP)
    ref.execute(0, 0, [y2], [m2], g2, a2, 1, DP)
    assert rel_l2(y1, y2) < TOL
    del t, m1, m2, y1, y2
    e = random_alm(lmax, cl=0.1 * cl, rng=rng)
    b = random_alm(lmax, cl=0.01 * cl, rng=rng)
    q1, u1, q2, u2 = (np.zeros(npix) for _ in range(4))
    sb.execute(1, 2, [e.copy(), b.copy()], [q1, u1], g1, a1, 1, DP)
    ref.execute(1, 2, [e.copy(), b.copy()], [q2, u2], g2, a2, 1, DP)
    assert rel_l2(q1, q2) < TOL and rel_l2(u1, u2) < TOL
    del q1, u1
    x1 = [np.zeros_like(e), np.zeros_like(e)]
    x2 = [np.zeros_like(e), np.zeros_like(e)]
    sb.execute(0, 2, x1, [q2, u2], g1, a1, 1, DP)
    ref.execute(0, 2, x2, [q2, u2], g2, a2, 1, DP)
    assert rel_l2(x1[0], x2[0]) < TOL and rel_l2(x1[1], x2[1]) < TOL


def test_results_are_bitwise_repeatable():
    nside, lmax = 64, 128
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    mp = np.random.default_rng(2).standard_normal(12 * nside * nside)
    outs = []
    for _ in range(2):
        o = [np.zeros(sb.nalm_triangular(lmax), np.complex128) for _ in range(2)]
        sb.execute(0, 2, o, [mp.copy(), mp[::-1].copy()], g, a, 1, DP)
        outs.append(o)
    assert all(np.array_equal(x, y) for x, y in zip(outs[0], outs[1]))


def test_device_pointer_entry_matches_host_entry():
    import torch
    nside, lmax = 32, 64
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    alm = random_alm(lmax, seed=4)
    host = np.zeros(12 * nside * nside)
    sb.execute(1, 0, [alm.copy()], [host], g, a, 1, DP)
    ta = torch.from_numpy(alm.view(np.float64).copy()).cuda()
    tm = torch.zeros(12 * nside * nside, dtype=torch.float64, device="cuda")
    sb.execute_device(1, 0, [ta], [tm], g, a, 1, DP)
    torch.cuda.synchronize()
    assert np.array_equal(tm.cpu().numpy(), host)


@pytest.mark.parametrize("spin", [0, 2])
def test_long_rings_match_reference(ref, spin):
    # rings too long for a shared-memory FFT (their buffers run in global
    # scratch): a power-of-two length 16384, a Bluestein length 8194
    # (8194/2 = 17 * 241) and a mixed-radix length 16380, with a few short
    # rings in the same geometry; both directions, weights, phi0 shifts
    lmax = 96
    nph = np.array([16384, 8194, 16380, 16384, 30, 8194, 64, 16380], np.int32)
    nr = len(nph)
    theta = np.linspace(0.3, 2.8, nr)
    ofs = np.concatenate([[0], np.cumsum(nph[:-1])]).astype(np.intp)
    st = np.ones(nr, np.int32)
    phi0 = np.linspace(0.0, 0.4, nr)
    w = np.linspace(0.5, 1.5, nr)
    g1 = sb.Geometry.general(nph, ofs, st, phi0, theta, w)
    g2 = ref.general(nph, ofs, st, phi0, theta, w)
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    npix = int(nph.sum())
    na = _nalm(1, spin)
    alms = [uniform_alm(lmax, seed=70 + i, spin=spin) for i in range(na)]
    m1 = [np.zeros(npix) for _ in range(na)]
    m2 = [np.zeros_like(x) for x in m1]
    sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, DP)
    ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, DP)
    for x, y in zip(m1, m2):
        assert rel_l2(x, y) < TOL
    rng = np.random.default_rng(spin)
    maps = [rng.standard_normal(npix) for _ in range(na)]
    o1 = [np.zeros(sb.nalm_triangular(lmax), np.complex128) for _ in range(na)]
    o2 = [x.copy() for x in o1]
    sb.execute(0, spin, o1, [x.copy() for x in maps], g1, a1, 1, DP)
    ref.execute(0, spin, o2, [x.copy() for x in maps], g2, a2, 1, DP)
    for x, y in zip(o1, o2):
        assert rel_l2(x, y) < TOL


def test_healpix_nside4096_matches_reference(ref):
    # Nside 4096 (rings up to 16384 pixels, the large-ring FFT path for the
    # equatorial belt and the longest polar rings) at a small lmax
    nside, lmax = 4096, 64
    o1, o2 = run_pair(ref, ("healpix", nside), lmax, lmax, 0, 1, seed=4)
    for x, y in zip(o1, o2):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_prime_ring_lengths_match_reference(ref, spin):
    # ring lengths with large prime factors: Bluestein with convolution
    # lengths 128 (odd number of radix-2 stages) and 256 (even), odd ring
    # lengths, a generic radix-37 pass; paired rings of different lengths,
    # phi0 shifts and weights; both directions against the reference
    nph = np.array([61, 127, 122, 254, 111, 64, 97, 194], np.int32)
    nr = len(nph)
    theta = np.linspace(0.2, np.pi - 0.2, nr)
    ofs = np.concatenate([[0], np.cumsum(nph)[:-1]])
    st = np.ones(nr, np.int32)
    phi0 = np.linspace(0.0, 0.7, nr)
    w = np.linspace(0.5, 1.5, nr) * 4 * np.pi / nph.sum()
    g1 = sb.Geometry.general(nph, ofs, st, phi0, theta, w)
    g2 = ref.general(nph, ofs, st, phi0, theta, w)
    lmax = 40
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    npix = int(nph.sum())
    na = _nalm(1, spin)
    alms = [uniform_alm(lmax, seed=40 + i, spin=spin) for i in range(na)]
    m1 = [np.zeros(npix) for _ in range(na)]
    m2 = [np.zeros(npix) for _ in range(na)]
    sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, DP)
    ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, DP)
    for x, y in zip(m1, m2):
        assert rel_l2(x, y) < TOL
    rng = np.random.default_rng(17)
    maps = [rng.standard_normal(npix) for _ in range(na)]
    b1 = [np.zeros_like(alms[0]) for _ in range(na)]
    b2 = [np.zeros_like(alms[0]) for _ in range(na)]
    sb.execute(0, spin, b1, [x.copy() for x in maps], g1, a1, 1, DP)
    ref.execute(0, spin, b2, [x.copy() for x in maps], g2, a2, 1, DP)
    for x, y in zip(b1, b2):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spin", [0, 2])
@pytest.mark.parametrize("flags", [DP, 0])
def test_register_bluestein_rings_match_reference(ref, spin, flags):
    # even rings whose half length has a large prime factor: Bluestein
    # convolution lengths 1024 (1018 = 2 * 509), 2048 (2004 = 4 * 3 * 167),
    # 4096 (2062 = 2 * 1031) and 8192 (4124 = 4 * 1031, the polar HEALPix
    # form 4i); long even rings of small factors that the register
    # convolution takes as well (2400 = 2 * 1200, 6000 = 2 * 3000); alias
    # folding (lmax above half the shorter rings), phi0 shifts, weights, an
    # interleaved stride-2 pair, an unpaired ring and a pair of unequal
    # lengths (which takes the size-class kernels); both directions, FP64
    # and single-precision I/O
    rings = [  # (nph, theta, phi0, stride)
        (1018, 0.7, 0.1, 1), (1018, np.pi - 0.7, 0.1, 1),
        (2004, 0.9, 0.0, 1), (2004, np.pi - 0.9, 0.0, 1),
        (2062, 1.1, 0.3, 1), (2062, np.pi - 1.1, 0.3, 1),
        (4124, 1.3, 0.05, 1), (4124, np.pi - 1.3, 0.05, 1),
        (1018, 1.45, 0.2, 2), (1018, np.pi - 1.45, 0.2, 2),
        (2004, np.pi / 2, 0.4, 1),
        (1018, 0.5, 0.0, 1), (2004, np.pi - 0.5, 0.0, 1),
        (2400, 0.35, 0.15, 1), (2400, np.pi - 0.35, 0.15, 1),
        (6000, 0.25, 0.0, 1), (6000, np.pi - 0.25, 0.0, 1),
    ]
    nph = np.array([r[0] for r in rings], np.int32)
    theta = np.array([r[1] for r in rings])
    phi0 = np.array([r[2] for r in rings])
    st = np.array([r[3] for r in rings], np.int32)
    ofs = np.zeros(len(rings), np.intp)
    pos = 0
    for i, r in enumerate(rings):
        if r[3] == 2 and i > 0 and rings[i - 1][3] == 2:
            ofs[i] = ofs[i - 1] + 1         # interleaved with the previous ring
            pos = ofs[i - 1] + 2 * r[0]
        else:
            ofs[i] = pos
            pos += r[0] * r[3]
    npix = int(pos)
    w = np.linspace(0.5, 1.5, len(rings)) * 4 * np.pi / npix
    g1 = sb.Geometry.general(nph, ofs, st, phi0, theta, w)
    g2 = ref.general(nph, ofs, st, phi0, theta, w)
    lmax = 1100
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    nreal = np.float64 if flags & DP else np.float32
    ncpx = np.complex128 if flags & DP else np.complex64
    tol = TOL if flags & DP else 1e-6
    na = _nalm(1, spin)
    alms = [uniform_alm(lmax, seed=90 + i, spin=spin).astype(ncpx) for i in range(na)]
    m1 = [np.zeros(npix, nreal) for _ in range(na)]
    m2 = [np.zeros(npix, nreal) for _ in range(na)]
    sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, flags)
    ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, flags)
    for x, y in zip(m1, m2):
        assert rel_l2(x, y) < tol
    rng = np.random.default_rng(23 + spin)
    maps = [rng.standard_normal(npix).astype(nreal) for _ in range(na)]
    b1 = [np.zeros(sb.nalm_triangular(lmax), ncpx) for _ in range(na)]
    b2 = [x.copy() for x in b1]
    sb.execute(0, spin, b1, [x.copy() for x in maps], g1, a1, 1, flags)
    ref.execute(0, spin, b2, [x.copy() for x in maps], g2, a2, 1, flags)
    for x, y in zip(b1, b2):
        assert rel_l2(x, y) < tol


@pytest.mark.parametrize("spin", [0, 2])
def test_healpix_nside512_lmax1024_both_directions(ref, spin):
    # Nside 512: the equatorial rings (2048 pixels) take the power-of-two
    # register FFT of length 1024 (the shortest), the polar rings the
    # register Bluestein lengths 1024 and 2048 and the size classes; both
    # directions against the reference at 1e-12
    for jtype in (1, 0):
        o1, o2 = run_pair(ref, ("healpix", 512), 1024, 1024, spin, jtype, seed=11 + spin)
        for x, y in zip(o1, o2):
            assert rel_l2(x, y) < TOL, (spin, jtype)


@pytest.mark.parametrize("spin", [0, 2])
def test_every_ring_length_1_to_4096_matches_reference(ref, spin):
    # the counterpart of the reference's ffttest (every length 1..4096): one
    # ring of each length, unpaired, at distinct colatitudes, phi0 shifts and
    # weights; lmax 64, so the short rings fold the phases and the long ones
    # take every FFT path (size classes with all radix mixes and Bluestein,
    # power-of-two rings, register Bluestein); both directions at 1e-12
    nph = np.arange(1, 4097, dtype=np.int32)
    nr = len(nph)
    theta = np.linspace(0.02, np.pi / 2 - 0.02, nr)
    ofs = np.concatenate([[0], np.cumsum(nph)[:-1]])
    st = np.ones(nr, np.int32)
    phi0 = np.linspace(0.0, 1.0, nr)
    w = np.linspace(0.5, 1.5, nr) * 4 * np.pi / nph.sum()
    g1 = sb.Geometry.general(nph, ofs, st, phi0, theta, w)
    g2 = ref.general(nph, ofs, st, phi0, theta, w)
    lmax = 64
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    npix = int(nph.sum())
    na = _nalm(1, spin)
    alms = [uniform_alm(lmax, seed=60 + i, spin=spin) for i in range(na)]
    m1 = [np.zeros(npix) for _ in range(na)]
    m2 = [np.zeros(npix) for _ in range(na)]
    sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, DP)
    ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, DP)
    for x, y in zip(m1, m2):
        assert rel_l2(x, y) < TOL
    rng = np.random.default_rng(29 + spin)
    maps = [rng.standard_normal(npix) for _ in range(na)]
    b1 = [np.zeros(sb.nalm_triangular(lmax), np.complex128) for _ in range(na)]
    b2 = [x.copy() for x in b1]
    sb.execute(0, spin, b1, [x.copy() for x in maps], g1, a1, 1, DP)
    ref.execute(0, spin, b2, [x.copy() for x in maps], g2, a2, 1, DP)
    for x, y in zip(b1, b2):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_ring_lengths_with_folding_at_high_lmax(ref, spin):
    # lmax 2100 folds the phases of every ring up to 4200 pixels: lengths
    # 1..4096 in steps of 7 plus the power-of-two and neighbouring lengths
    # (the register FFT classes then take folded rings: 4096 pixels goes to
    # the register Bluestein convolution of length 4096), unpaired rings,
    # phi0 shifts and weights; both directions at 1e-12
    nph = np.unique(np.concatenate([np.arange(1, 4097, 7), [2047, 2048, 2049, 4094, 4095, 4096]]))
    nph = nph.astype(np.int32)
    nr = len(nph)
    theta = np.linspace(0.3, np.pi / 2 - 0.02, nr)
    ofs = np.concatenate([[0], np.cumsum(nph)[:-1]])
    st = np.ones(nr, np.int32)
    phi0 = np.linspace(0.0, 0.9, nr)
    w = np.linspace(0.5, 1.5, nr) * 4 * np.pi / nph.sum()
    g1 = sb.Geometry.general(nph, ofs, st, phi0, theta, w)
    g2 = ref.general(nph, ofs, st, phi0, theta, w)
    lmax = 2100
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    npix = int(nph.sum())
    na = _nalm(1, spin)
    alms = [uniform_alm(lmax, seed=70 + i, spin=spin) for i in range(na)]
    m1 = [np.zeros(npix) for _ in range(na)]
    m2 = [np.zeros(npix) for _ in range(na)]
    sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, DP)
    ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, DP)
    for x, y in zip(m1, m2):
        assert rel_l2(x, y) < TOL
    rng = np.random.default_rng(31 + spin)
    maps = [rng.standard_normal(npix) for _ in range(na)]
    b1 = [np.zeros(sb.nalm_triangular(lmax), np.complex128) for _ in range(na)]
    b2 = [x.copy() for x in b1]
    sb.execute(0, spin, b1, [x.copy() for x in maps], g1, a1, 1, DP)
    ref.execute(0, spin, b2, [x.copy() for x in maps], g2, a2, 1, DP)
    for x, y in zip(b1, b2):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_negative_and_interleaved_strides_match_reference(ref, spin):
    # rings stored backwards (stride -1) and interleaved pairs (strides +2 and
    # -2 over one pixel range), for a short ring, a folded mid-length ring,
    # a 4096-pixel ring (which then leaves the power-of-two class for the
    # register Bluestein one) and an 8188-pixel polar-style ring; both
    # directions at 1e-12
    specs = [(30, 1), (30, -1), (1000, -1), (4096, -1), (4096, 1), (8188, -1), (518, 2), (518, -2)]
    nph = np.array([n for n, _ in specs], np.int32)
    st = np.array([s for _, s in specs], np.int32)
    ofs = np.zeros(len(specs), np.intp)
    pos = 0
    i = 0
    while i < len(specs):
        n, s = specs[i]
        if abs(s) == 2:
            # this ring and the next share 2n pixels: +2 from pos, -2 from the end
            ofs[i] = pos
            ofs[i + 1] = pos + 2 * n - 1
            pos += 2 * n
            i += 2
            continue
        ofs[i] = pos if s > 0 else pos + n - 1
        pos += n
        i += 1
    npix = int(pos)
    cover = np.zeros(npix, int)
    for k in range(len(specs)):
        cover[ofs[k] + st[k] * np.arange(nph[k])] += 1
    assert cover.min() == 1 and cover.max() == 1
    nr = len(specs)
    theta = np.linspace(0.25, 1.45, nr)
    phi0 = np.linspace(0.0, 0.6, nr)
    w = np.linspace(0.5, 1.5, nr)
    g1 = sb.Geometry.general(nph, ofs, st, phi0, theta, w)
    g2 = ref.general(nph, ofs, st, phi0, theta, w)
    lmax = 700
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    na = _nalm(1, spin)
    alms = [uniform_alm(lmax, seed=80 + i, spin=spin) for i in range(na)]
    m1 = [np.zeros(npix) for _ in range(na)]
    m2 = [np.zeros(npix) for _ in range(na)]
    sb.execute(1, spin, [x.copy() for x in alms], m1, g1, a1, 1, DP)
    ref.execute(1, spin, [x.copy() for x in alms], m2, g2, a2, 1, DP)
    for x, y in zip(m1, m2):
        assert rel_l2(x, y) < TOL
    rng = np.random.default_rng(41 + spin)
    maps = [rng.standard_normal(npix) for _ in range(na)]
    b1 = [np.zeros(sb.nalm_triangular(lmax), np.complex128) for _ in range(na)]
    b2 = [x.copy() for x in b1]
    sb.execute(0, spin, b1, [x.copy() for x in maps], g1, a1, 1, DP)
    ref.execute(0, spin, b2, [x.copy() for x in maps], g2, a2, 1, DP)
    for x, y in zip(b1, b2):
        assert rel_l2(x, y) < TOL
