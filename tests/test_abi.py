"""Host-side checks of the C-ABI library (no GPU needed): it loads, exports
every function the public headers declare, builds the same geometries and
a_lm layouts as the reference, and reports bad arguments the way the
reference does (message + exit(1) by default, or an error string when abort
is switched off)."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import sharp_b200 as sb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^(?!\s*static)[\w\s\*]*?\b(sharp_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert "sharp_execute" in names and "sharp_b200_execute_device" in names
    lib = ctypes.CDLL(sb.LIB_PATH, mode=os.RTLD_LOCAL)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # the inline helpers stay inline, as in the reference headers
    assert "sharp_make_healpix_geom_info" not in names


def _pairs(geom):
    g = geom.ptr.contents
    out = []
    for i in range(g.npairs):
        p = g.pair[i]
        out.append(tuple((r.theta, r.phi0, r.weight, r.cth, r.sth, r.ofs, r.nph, r.stride)
                         for r in (p.r1, p.r2) if r.nph > 0))
    return out


def _compare_geoms(ours, theirs, wtol, ctol=1e-15):
    """Ring indexing (ofs, nph, stride) must be identical; theta/phi0 within
    an ulp (the reference is built with -ffast-math), cos/sin within 1e-15
    absolute (a 1-ulp theta near the poles moves sin(theta) by more than an
    ulp), weights within ``wtol`` relative."""
    a, b = _pairs(ours), _pairs(theirs)
    assert len(a) == len(b)
    for pa, pb in zip(a, b):
        assert len(pa) == len(pb)
        for ra, rb in zip(pa, pb):
            assert ra[5:] == rb[5:]
            # theta = acos(cth) is ill-conditioned near the poles: check it
            # through cos/sin there
            assert abs(ra[1] - rb[1]) <= 5e-16 * abs(rb[1])
            assert abs(ra[0] - rb[0]) * max(rb[4], 1e-300) <= ctol
            assert abs(ra[2] - rb[2]) <= wtol * abs(rb[2])
            assert np.allclose(ra[3:5], rb[3:5], rtol=0, atol=ctol)


@pytest.fixture(scope="module")
def ref():
    r = pytest.importorskip("ref")
    if not r.available():
        pytest.skip("reference library not built (make -C oracle)")
    return r


@pytest.mark.parametrize("nside", [1, 2, 3, 16, 64, 1024])
def test_healpix_geometry_matches_reference(ref, nside):
    w = np.linspace(0.5, 1.5, 2 * nside)
    _compare_geoms(sb.Geometry.healpix(nside), ref.healpix(nside), 4e-16)
    _compare_geoms(sb.Geometry.healpix(nside, weight=w), ref.healpix(nside, weight=w), 4e-16)
    _compare_geoms(sb.Geometry.healpix(nside, stride=3), ref.healpix(nside, stride=3), 4e-16)


# Gauss-Legendre weights near the poles are 2/((1-x^2) P_n'(x)^2) with a
# cancellation in P_n'; two correct builds differ there by up to ~1e-10.
@pytest.mark.parametrize("kind,nr,nphi", [("gauss", 51, 102), ("gauss", 128, 256),
                                          ("gauss", 1025, 2049), ("fejer1", 65, 128),
                                          ("fejer1", 64, 127), ("fejer2", 63, 128),
                                          ("cc", 65, 128), ("cc", 64, 129), ("mw", 33, 65)])
def test_grid_geometry_matches_reference(ref, kind, nr, nphi):
    _compare_geoms(sb.Geometry.grid(kind, nr, nphi, 0.3, 1, nphi),
                   ref.grid(kind, nr, nphi, 0.3, 1, nphi), 1e-9 if kind == "gauss" else 1e-12,
                   ctol=2e-14)


def test_general_geometry_pairs_like_reference(ref):
    rng = np.random.default_rng(5)
    nr = 40
    theta = np.sort(rng.uniform(0.05, np.pi - 0.05, nr // 2))
    theta = np.concatenate([theta, np.pi - theta[:10]])
    nph = rng.integers(3, 30, len(theta)).astype(np.int32)
    ofs = np.concatenate([[0], np.cumsum(nph)[:-1]])
    st = np.ones(len(theta), np.int32)
    phi0 = rng.uniform(0, 1, len(theta))
    w = rng.uniform(0.5, 1, len(theta))
    _compare_geoms(sb.Geometry.general(nph, ofs, st, phi0, theta, w),
                   ref.general(nph, ofs, st, phi0, theta, w), 0)


def test_alm_layouts(ref):
    for lmax, mmax in ((10, 10), (20, 7)):
        ours = sb.AlmInfo.triangular(lmax, mmax).ptr.contents
        # keep the owners alive while reading the structs
        o1 = sb.AlmInfo.triangular(lmax, mmax)
        r1 = ref.triangular(lmax, mmax)
        a, b = o1.ptr.contents, r1.ptr.contents
        assert (a.lmax, a.nm, a.stride) == (b.lmax, b.nm, b.stride)
        assert [a.mvstart[i] for i in range(a.nm)] == [b.mvstart[i] for i in range(b.nm)]
        o2 = sb.AlmInfo.rectangular(lmax, mmax, 2)
        assert [o2.ptr.contents.mvstart[i] for i in range(mmax + 1)] == \
            [2 * m * (lmax + 1) for m in range(mmax + 1)]
        assert o1.index(lmax, mmax) == sb.nalm_triangular(lmax, mmax) - 1
        del ours


def test_bad_arguments_report_errors_without_abort():
    sb.set_abort_on_error(False)
    try:
        g = sb.Geometry.healpix(4)
        a = sb.AlmInfo.triangular(8)
        alm = [np.zeros(sb.nalm_triangular(8), np.complex128)]
        mp = [np.zeros(192)]
        with pytest.raises(sb.SharpError, match="bad number of simultaneous transforms"):
            sb.execute(sb.SHARP_ALM2MAP, 0, alm, mp, g, a, 0)
        with pytest.raises(sb.SharpError, match="bad number of simultaneous transforms"):
            sb.execute(sb.SHARP_ALM2MAP, 0, alm, mp, g, a, 101)
        with pytest.raises(sb.SharpError, match="bad spin"):
            sb.execute(sb.SHARP_ALM2MAP, 9, alm * 2, mp * 2, g, a, 1)
        bad = sb.AlmInfo.general(8, [0, 1, 1], [0, 8, 16])
        with pytest.raises(sb.SharpError, match="duplicate m value"):
            sb.execute(sb.SHARP_ALM2MAP, 0, alm, mp, g, bad, 1)
        gap = sb.AlmInfo.general(8, [0, 2], [0, 8])
        with pytest.raises(sb.SharpError, match="not all m values are present"):
            sb.execute(sb.SHARP_ALM2MAP, 0, alm, mp, g, gap, 1)
        with pytest.raises(sb.SharpError, match="bad ring size"):
            sb.execute(sb.SHARP_ALM2MAP, 0, alm, mp, g, a, 1, sb.SHARP_DP | sb.SHARP_NO_FFT)
        with pytest.raises(sb.SharpError, match="ADJOINT"):
            sb.execute(sb.SHARP_ALM2MAP_DERIV1, 1, alm, mp * 2, g, a, 1,
                       sb.SHARP_DP | sb.SHARP_ADJOINT)
        assert sb.last_error() == ""
    finally:
        sb.set_abort_on_error(os.environ.get("SHARP_B200_ABORT_ON_ERROR", "1") != "0")


def test_batch_validates_jobs_before_running():
    # every job is checked before the first one runs: a bad job anywhere in
    # the list fails the call with the single-job message
    sb.set_abort_on_error(False)
    try:
        g = sb.Geometry.healpix(4)
        a = sb.AlmInfo.triangular(8)
        alm = [np.zeros(sb.nalm_triangular(8), np.complex128)]
        mp = [np.zeros(192)]
        good = (sb.SHARP_ALM2MAP, 0, alm, mp, g, a, 1, sb.SHARP_DP)
        bad = (sb.SHARP_ALM2MAP, 0, alm, mp, g, a, 0, sb.SHARP_DP)
        with pytest.raises(sb.SharpError, match="bad number of simultaneous transforms"):
            sb.execute_batch([good, bad])
        assert sb.execute_batch([]) == (0, 0)
    finally:
        sb.set_abort_on_error(os.environ.get("SHARP_B200_ABORT_ON_ERROR", "1") != "0")


def test_bad_arguments_abort_like_reference_by_default():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np, sharp_b200 as sb\n"
        "g = sb.Geometry.healpix(2); a = sb.AlmInfo.triangular(4)\n"
        "sb.execute(0, 0, [np.zeros(15, complex)], [np.zeros(48)], g, a, 0)\n"
        "print('not reached')\n") % os.path.join(ROOT, "planck-levels_b200")
    env = dict(os.environ)
    env.pop("SHARP_B200_ABORT_ON_ERROR", None)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env)
    assert r.returncode == 1
    assert "bad number of simultaneous transforms" in r.stderr
    assert "not reached" not in r.stdout
