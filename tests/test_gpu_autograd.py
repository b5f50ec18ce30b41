"""Differentiation through the adjoint kernels (SHARP_ADJOINT) and the
device-resident Healpix_cxx pipelines.

The chi^2 loss L(a) = 1/2 ||W (alm2map(a) - d)||^2 at Nside 512, lmax 1024,
spin 0 + 2 (T, E, B): its gradient from the torch.autograd.Function must
match central finite differences along 32 random unit directions in a_lm
space (m = 0 imaginary parts held at zero) within 1e-6 relative."""
import numpy as np
import pytest

import sharp_b200 as sb
from helpers import cl_spectrum, random_alm, rel_l2

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def test_chi2_gradient_matches_central_differences():
    torch = _torch()
    from sharp_b200 import autograd as sa
    nside, lmax = 512, 1024
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    npix = 12 * nside * nside
    rng = np.random.default_rng(11)
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

    def loss(alms):
        mT = sa.alm2map(g, a, 0, alms[0])
        mQ, mU = sa.alm2map(g, a, 2, alms[1], alms[2])
        return 0.5 * sum(((w * (m - dd)) ** 2).sum() for w, m, dd in zip(W, (mT, mQ, mU), d))

    xs = [x.clone().requires_grad_(True) for x in x0]
    L = loss(xs)
    L.backward()
    grads = [x.grad.detach() for x in xs]
    # gradient of Im a_l0 must vanish (not an input of Y)
    for gr in grads:
        assert torch.all(gr[: lmax + 1].imag == 0)
    worst = 0.0
    for k in range(32):
        v = [torch.from_numpy(rng.standard_normal(x.numel()) + 1j * rng.standard_normal(x.numel())).to(dev)
             for x in x0]
        for vv in v:
            vv[: lmax + 1] = vv[: lmax + 1].real.to(vv.dtype)
        nrm = torch.sqrt(sum((vv.real ** 2 + vv.imag ** 2).sum() for vv in v))
        v = [vv / nrm for vv in v]
        h = 1e-3
        with torch.no_grad():
            lp = loss([x + h * vv for x, vv in zip(x0, v)])
            lm = loss([x - h * vv for x, vv in zip(x0, v)])
        fd = float((lp - lm) / (2 * h))
        an = float(sum((gr.real * vv.real + gr.imag * vv.imag).sum() for gr, vv in zip(grads, v)))
        worst = max(worst, abs(fd - an) / max(abs(fd), 1e-300))
    assert worst < 1e-6, worst


def test_map2alm_gradient_matches_central_differences():
    torch = _torch()
    from sharp_b200 import autograd as sa
    nside, lmax = 64, 128
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    npix = 12 * nside * nside
    rng = np.random.default_rng(5)
    target = [torch.from_numpy(random_alm(lmax, rng=rng)).cuda() for _ in range(2)]
    m0 = [torch.from_numpy(rng.standard_normal(npix)).cuda() for _ in range(2)]

    def loss(maps):
        e, b = sa.map2alm(g, a, 2, *maps)
        return 0.5 * sum(((x - t).abs() ** 2).sum() for x, t in zip((e, b), target))

    ms = [m.clone().requires_grad_(True) for m in m0]
    loss(ms).backward()
    for k in range(8):
        v = [torch.from_numpy(rng.standard_normal(npix)).cuda() for _ in range(2)]
        nrm = torch.sqrt(sum((vv ** 2).sum() for vv in v))
        v = [vv / nrm for vv in v]
        h = 1e-3
        with torch.no_grad():
            fd = float((loss([m + h * vv for m, vv in zip(m0, v)]) -
                        loss([m - h * vv for m, vv in zip(m0, v)])) / (2 * h))
        an = float(sum((m.grad * vv).sum() for m, vv in zip(ms, v)))
        assert abs(fd - an) < 1e-6 * abs(fd), (k, fd, an)


def test_device_pipelines_match_reference():
    torch = _torch()
    import ref
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    from sharp_b200 import healpix as hp
    nside, lmax = 64, 128
    g2, a2 = ref.healpix(nside), ref.triangular(lmax, lmax)
    npix = 12 * nside * nside
    rng = np.random.default_rng(8)
    t, e, b = (random_alm(lmax, rng=rng) for _ in range(3))
    # alm2map_pol on the device vs the reference's spin-0 + spin-2 jobs
    mT, mQ, mU = (torch.zeros(npix, dtype=torch.float64, device="cuda") for _ in range(3))
    hp.alm2map_pol(*(torch.from_numpy(x).cuda() for x in (t, e, b)), mT, mQ, mU, lmax)
    r = [np.zeros(npix) for _ in range(3)]
    ref.execute(1, 0, [t.copy()], [r[0]], g2, a2, 1, 16)
    ref.execute(1, 2, [e.copy(), b.copy()], [r[1], r[2]], g2, a2, 1, 16)
    for x, y in zip((mT, mQ, mU), r):
        assert rel_l2(x.cpu().numpy(), y) < 1e-12
    # map2alm_pol_iter with 3 Jacobi sweeps vs the same loop on the reference
    at, ae, ab = (torch.zeros(len(t), dtype=torch.complex128, device="cuda") for _ in range(3))
    hp.map2alm_pol_iter(*(torch.from_numpy(x).cuda() for x in r), at, ae, ab, lmax, 3)
    ra = [np.zeros_like(t) for _ in range(3)]
    ref.execute(0, 0, [ra[0]], [r[0].copy()], g2, a2, 1, 16)
    ref.execute(0, 2, [ra[1], ra[2]], [r[1].copy(), r[2].copy()], g2, a2, 1, 16)
    for _ in range(3):
        w = [np.zeros(npix) for _ in range(3)]
        ref.execute(1, 0, [ra[0].copy()], [w[0]], g2, a2, 1, 16)
        ref.execute(1, 2, [ra[1].copy(), ra[2].copy()], [w[1], w[2]], g2, a2, 1, 16)
        res = [x - y for x, y in zip(r, w)]
        ref.execute(0, 0, [ra[0]], [res[0]], g2, a2, 1, 16 | 32)
        ref.execute(0, 2, [ra[1], ra[2]], [res[1], res[2]], g2, a2, 1, 16 | 32)
    for x, y in zip((at, ae, ab), ra):
        assert rel_l2(x.cpu().numpy(), y) < 1e-12
    # first derivatives
    m0, dth, dph = (torch.zeros(npix, dtype=torch.float64, device="cuda") for _ in range(3))
    hp.alm2map_der1(torch.from_numpy(t).cuda(), m0, dth, dph, lmax)
    d1, d2 = np.zeros(npix), np.zeros(npix)
    ref.execute(4, 1, [t.copy()], [d1, d2], g2, a2, 1, 16)
    assert rel_l2(dth.cpu().numpy(), d1) < 1e-12 and rel_l2(dph.cpu().numpy(), d2) < 1e-12
