"""Device-resident Healpix_cxx program bodies and the library pieces they
use, against the reference libsharp:

* SHARP_SUBTRACT: output -= result, bit for bit the negated SHARP_ADD;
* alm2map_cxx, anafast_cxx and smoothing_cxx (sharp_b200.healpix) with
  Gaussian beams, pixel windows, monopole handling and undefined pixels,
  against the same steps restated here in numpy around reference transforms
  (Healpix_cxx/alm2map_cxx_module.cc:80-127, anafast_cxx_module.cc:55-127,
  smoothing_cxx_module.cc:49-115, alm_powspec_tools.cc:250-299);
* gradients with precision="mixed" (SHARP_MIXED forward and adjoint) against
  central finite differences of the FP64 loss, and the mixed adjoint
  transforms against the reference's SHARP_Yt / SHARP_WY;
* sharp_b200_check_device_errors after SHARP_MIXED device-pointer work.
"""
import math

import numpy as np
import pytest

import sharp_b200 as sb
from helpers import cl_spectrum, random_alm, rel_l2, uniform_alm

pytestmark = pytest.mark.gpu
DP, MIXED, SUB = sb.SHARP_DP, sb.SHARP_MIXED, sb.SHARP_SUBTRACT
FOURPI = 12.56637061435917295385057353311801153679   # cxxsupport/lsconstants.h:38
FWHM2SIGMA = 1.0 / 2.3548200450309493                # lsconstants.h:56-57
UNDEF = -1.6375e30


@pytest.fixture(scope="module")
def ref():
    import ref as r
    if not r.available():
        pytest.skip("reference library not built (make -C oracle)")
    return r


@pytest.mark.parametrize("spin", [0, 2])
@pytest.mark.parametrize("mixed", [False, True])
def test_subtract_flag_is_negated_add(spin, mixed):
    nside, lmax = 32, 64
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    flags = DP | (MIXED if mixed else 0)
    nc = 1 if spin == 0 else 2
    npix = 12 * nside * nside
    rng = np.random.default_rng(3 + spin)
    alms = [uniform_alm(lmax, seed=20 + i, spin=spin) for i in range(nc)]
    plain = [np.zeros(npix) for _ in range(nc)]
    sb.execute(1, spin, [x.copy() for x in alms], plain, g, a, 1, flags)
    init = [rng.standard_normal(npix) for _ in range(nc)]
    out = [x.copy() for x in init]
    sb.execute(1, spin, [x.copy() for x in alms], out, g, a, 1, flags | SUB)
    for o, i0, p in zip(out, init, plain):
        assert np.array_equal(o, i0 - p)
    maps = [rng.standard_normal(npix) for _ in range(nc)]
    plain = [np.zeros_like(alms[0]) for _ in range(nc)]
    sb.execute(0, spin, plain, [x.copy() for x in maps], g, a, 1, flags)
    out = [x.copy() for x in alms]
    sb.execute(0, spin, out, [x.copy() for x in maps], g, a, 1, flags | SUB)
    for o, i0, p in zip(out, alms, plain):
        assert np.array_equal(o, i0 - p)
    with pytest.raises(sb.SharpError):
        sb.execute(0, spin, out, [x.copy() for x in maps], g, a, 1, flags | SUB | sb.SHARP_ADD)


# --- reference-side restatements ------------------------------------------
def _lidx(lmax):
    return np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])


def _scale_l(alm, f, lmax):
    # Alm::ScaleL, Healpix_cxx/alm.h:122-129
    ff = f[_lidx(lmax)]
    alm.real *= ff
    alm.imag *= ff


def _gauss(fwhm, lmax, pol=False):
    # smoothWithGauss, alm_powspec_tools.cc:250-283
    fct = 1 if fwhm >= 0 else -1
    sigma = fwhm * FWHM2SIGMA
    l = np.arange(lmax + 1, dtype=np.float64)
    gb = np.exp(-.5 * fct * l * (l + 1) * sigma * sigma)
    return gb * math.exp(2 * fct * sigma * sigma) if pol else gb


def _defined(x):
    return np.abs(x - UNDEF) > 1e-5 * abs(UNDEF)   # approx(), cxxsupport/math_utils.h:43


def _ref_iter(ref, g, a, spin_maps, lmax, niter):
    """map2alm_iter / map2alm_pol_iter (alm_healpix_tools.cc:73-85, 239-265) on
    the reference: spin_maps = [(spin, [maps])]; returns the a_lm lists."""
    nalm = (lmax + 1) * (lmax + 2) // 2
    out = []
    for spin, maps in spin_maps:
        al = [np.zeros(nalm, np.complex128) for _ in maps]
        ref.execute(0, spin, al, [x.copy() for x in maps], g, a, 1, DP)
        out.append(al)
    for _ in range(niter):
        for (spin, maps), al in zip(spin_maps, out):
            w = [np.zeros_like(maps[0]) for _ in maps]
            ref.execute(1, spin, [x.copy() for x in al], w, g, a, 1, DP)
            res = [x - y for x, y in zip(maps, w)]
            ref.execute(0, spin, al, res, g, a, 1, DP | sb.SHARP_ADD)
    return out


def test_alm2map_cxx_matches_reference(ref):
    import torch
    from sharp_b200 import healpix as hp
    nside, lmax = 64, 128
    g2, a2 = ref.healpix(nside), ref.triangular(lmax, lmax)
    npix = 12 * nside * nside
    t, e, b = (uniform_alm(lmax, seed=300 + i, spin=2 * (i > 0)) for i in range(3))
    fwhm = 30.0 * math.pi / 10800.0
    # pixel windows are read from files by the program; smooth stand-ins here
    l = np.arange(lmax + 1)
    wt, wp = np.exp(-l / 400.0), np.exp(-l / 300.0)
    dev = [torch.from_numpy(x).cuda() for x in (t, e, b)]
    mT, mQ, mU = (torch.zeros(npix, dtype=torch.float64, device="cuda") for _ in range(3))
    hp.alm2map_cxx(dev[0], mT, lmax, fwhm=fwhm, pixwin=wt, almG=dev[1], almC=dev[2],
                   mapQ=mQ, mapU=mU, pixwin_pol=wp)
    assert np.array_equal(dev[0].cpu().numpy(), t)           # inputs untouched
    # alm2map_cxx_module.cc:108-121 with the reference transforms
    rt, re_, rb = t.copy(), e.copy(), b.copy()
    _scale_l(rt, _gauss(fwhm, lmax), lmax)
    _scale_l(re_, _gauss(fwhm, lmax, True), lmax)
    _scale_l(rb, _gauss(fwhm, lmax, True), lmax)
    _scale_l(rt, wt, lmax)
    _scale_l(re_, wp, lmax)
    _scale_l(rb, wp, lmax)
    offset = rt[0].real / math.sqrt(FOURPI)
    rt[0] = 0
    r = [np.zeros(npix) for _ in range(3)]
    ref.execute(1, 0, [rt], [r[0]], g2, a2, 1, DP)
    ref.execute(1, 2, [re_, rb], [r[1], r[2]], g2, a2, 1, DP)
    r[0] += offset
    for x, y in zip((mT, mQ, mU), r):
        assert rel_l2(x.cpu().numpy(), y) < 1e-12
    # the spin-0 branch alone, cosine window instead of a pixel window
    m0 = torch.zeros(npix, dtype=torch.float64, device="cuda")
    hp.alm2map_cxx(dev[0], m0, lmax, fwhm=fwhm, cosine=(40, 100))
    rt = t.copy()
    _scale_l(rt, _gauss(fwhm, lmax), lmax)
    cw = np.array([1.0 if i < 40 else (1 + math.cos(math.pi * (i - 40) / 60.0)) / 2
                   if i < 100 else 0.0 for i in range(lmax + 1)])
    _scale_l(rt, cw, lmax)
    off = rt[0].real / math.sqrt(FOURPI)
    rt[0] = 0
    r0 = np.zeros(npix)
    ref.execute(1, 0, [rt], [r0], g2, a2, 1, DP)
    assert rel_l2(m0.cpu().numpy(), r0 + off) < 1e-12


def test_anafast_and_smoothing_match_reference(ref):
    import torch
    from sharp_b200 import healpix as hp
    nside, lmax = 64, 128
    g2, a2 = ref.healpix(nside), ref.triangular(lmax, lmax)
    npix = 12 * nside * nside
    rng = np.random.default_rng(12)
    maps = [rng.standard_normal(npix) + (3.0 if i == 0 else 0.0) for i in range(3)]
    bad = rng.choice(npix, 40, replace=False)
    for x in maps:
        x[bad[:20]] = UNDEF
    maps[0][bad[20:]] = UNDEF
    nalm = (lmax + 1) * (lmax + 2) // 2
    # anafast_cxx_module.cc:95-117, polarised, monopole removal, 2 sweeps
    dm = [torch.from_numpy(x).cuda() for x in maps]
    at, ag, ac = (torch.zeros(nalm, dtype=torch.complex128, device="cuda") for _ in range(3))
    hp.anafast_cxx(dm[0], at, lmax, num_iter=2, remove_monopole=True, mapQ=dm[1], mapU=dm[2],
                   almG=ag, almC=ac)
    assert np.array_equal(dm[0].cpu().numpy(), maps[0], equal_nan=True)
    r = [x.copy() for x in maps]
    ok = _defined(r[0])
    avg = r[0][ok].sum() / ok.sum()
    r[0][ok] -= avg
    for x in r:
        x[~_defined(x)] = 0.0
    (rt,), (rg, rc) = _ref_iter(ref, g2, a2, [(0, [r[0]]), (2, [r[1], r[2]])], lmax, 2)
    rt[0] += avg * math.sqrt(FOURPI)
    for x, y in zip((at, ag, ac), (rt, rg, rc)):
        assert rel_l2(x.cpu().numpy(), y) < 1e-12
    # smoothing_cxx_module.cc:61-85, spin 0, 1 sweep, 20 arcmin
    fwhm = 20.0 * math.pi / 10800.0
    sm = torch.from_numpy(maps[0].copy()).cuda()
    hp.smoothing_cxx(sm, lmax, fwhm, num_iter=1)
    r0 = maps[0].copy()
    ok = _defined(r0)
    avg = r0[ok].sum() / ok.sum()
    r0[ok] -= avg
    r0[~ok] = 0.0
    (ra,), = _ref_iter(ref, g2, a2, [(0, [r0])], lmax, 1)
    _scale_l(ra, _gauss(fwhm, lmax), lmax)
    out = np.zeros(npix)
    ref.execute(1, 0, [ra], [out], g2, a2, 1, DP)
    out += avg
    assert rel_l2(sm.cpu().numpy(), out) < 1e-12


def test_mixed_chi2_gradient_matches_central_differences():
    # config 3 in mixed precision: the gradient from the SHARP_MIXED forward
    # and adjoint transforms against central differences of the FP64 loss
    import torch
    from sharp_b200 import autograd as sa
    nside, lmax = 512, 1024
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    npix = 12 * nside * nside
    rng = np.random.default_rng(13)
    cl = cl_spectrum(lmax, beam_arcmin=5.0)
    dev = "cuda"
    true = [torch.from_numpy(random_alm(lmax, cl=f * cl, rng=rng)).to(dev) for f in (1.0, 0.1, 0.01)]
    with torch.no_grad():
        dT = sa.alm2map(g, a, 0, true[0])
        dQ, dU = sa.alm2map(g, a, 2, true[1], true[2])
    noise = [0.1 * float(x.std()) * torch.from_numpy(rng.standard_normal(npix)).to(dev)
             for x in (dT, dQ, dU)]
    d = [dT + noise[0], dQ + noise[1], dU + noise[2]]
    W = [torch.from_numpy(rng.uniform(0.5, 2.0, npix)).to(dev) for _ in range(3)]
    x0 = [torch.from_numpy(random_alm(lmax, cl=f * cl, rng=rng)).to(dev) for f in (1.0, 0.1, 0.01)]

    def loss(alms, precision):
        mT = sa.alm2map(g, a, 0, alms[0], precision=precision)
        mQ, mU = sa.alm2map(g, a, 2, alms[1], alms[2], precision=precision)
        return 0.5 * sum(((w * (m - dd)) ** 2).sum() for w, m, dd in zip(W, (mT, mQ, mU), d))

    xs = [x.clone().requires_grad_(True) for x in x0]
    loss(xs, "mixed").backward()
    grads = [x.grad.detach() for x in xs]
    for gr in grads:
        assert torch.all(gr[: lmax + 1].imag == 0)
    worst = 0.0
    for _ in range(32):
        v = [torch.from_numpy(rng.standard_normal(x.numel()) + 1j * rng.standard_normal(x.numel())).to(dev)
             for x in x0]
        for vv in v:
            vv[: lmax + 1] = vv[: lmax + 1].real.to(vv.dtype)
        nrm = torch.sqrt(sum((vv.real ** 2 + vv.imag ** 2).sum() for vv in v))
        v = [vv / nrm for vv in v]
        h = 1e-3
        with torch.no_grad():
            lp = loss([x + h * vv for x, vv in zip(x0, v)], "fp64")
            lm = loss([x - h * vv for x, vv in zip(x0, v)], "fp64")
        fd = float((lp - lm) / (2 * h))
        an = float(sum((gr.real * vv.real + gr.imag * vv.imag).sum() for gr, vv in zip(grads, v)))
        worst = max(worst, abs(fd - an) / max(abs(fd), 1e-300))
    print(f"mixed-precision gradient vs central differences: worst relative error {worst:.2e}")
    assert worst < 1e-6, worst


@pytest.mark.parametrize("spin", [0, 2])
def test_mixed_adjoint_matches_reference_transpose_types(ref, spin):
    # SHARP_ADJOINT | SHARP_MIXED of alm2map is Yt, of map2alm is WY: against
    # the reference's own SHARP_Yt and SHARP_WY jobs within the 1e-6 bar
    nside, lmax = 128, 256
    g1, g2 = sb.Geometry.healpix(nside), ref.healpix(nside)
    a1, a2 = sb.AlmInfo.triangular(lmax), ref.triangular(lmax, lmax)
    nc = 1 if spin == 0 else 2
    npix = 12 * nside * nside
    rng = np.random.default_rng(60 + spin)
    maps = [rng.standard_normal(npix) for _ in range(nc)]
    y1 = [np.zeros(sb.nalm_triangular(lmax), np.complex128) for _ in range(nc)]
    y2 = [x.copy() for x in y1]
    sb.execute(sb.SHARP_ALM2MAP, spin, y1, [x.copy() for x in maps], g1, a1, 1,
               DP | MIXED | sb.SHARP_ADJOINT)
    ref.execute(sb.SHARP_Yt, spin, y2, [x.copy() for x in maps], g2, a2, 1, DP)
    for x, y in zip(y1, y2):
        assert rel_l2(x, y) < 1e-6
    alms = [uniform_alm(lmax, seed=70 + i, spin=spin) for i in range(nc)]
    w1 = [np.zeros(npix) for _ in range(nc)]
    w2 = [np.zeros(npix) for _ in range(nc)]
    sb.execute(sb.SHARP_MAP2ALM, spin, [x.copy() for x in alms], w1, g1, a1, 1,
               DP | MIXED | sb.SHARP_ADJOINT)
    ref.execute(sb.SHARP_WY, spin, [x.copy() for x in alms], w2, g2, a2, 1, DP)
    for x, y in zip(w1, w2):
        assert rel_l2(x, y) < 1e-6


def test_check_device_errors_after_mixed_device_work():
    import torch
    nside, lmax = 64, 128
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    alm = torch.from_numpy(uniform_alm(lmax, seed=5).view(np.float64).copy()).cuda()
    mp = torch.zeros(12 * nside * nside, dtype=torch.float64, device="cuda")
    sb.execute_device(sb.SHARP_ALM2MAP, 0, [alm], [mp], g, a, 1, DP | MIXED)
    sb.check_device_errors()
    assert sb.last_error() == ""
    assert float(mp.abs().max()) > 0
