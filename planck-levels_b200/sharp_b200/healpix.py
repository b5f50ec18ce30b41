"""Device-resident counterparts of Healpix_cxx's alm_healpix_tools.

Same names and argument meaning as zonca/planck-levelS
Healpix_cxx/alm_healpix_tools.{h,cc}, on torch CUDA tensors: a_lm are
complex128 tensors in the triangular m-major layout (Alm<T> order), maps are
float64 tensors in HEALPix RING order.  Everything stays in HBM between the
transform calls, including the Jacobi iterations of map2alm_iter.

    alm2map              alm_healpix_tools.cc:334-343
    map2alm              alm_healpix_tools.cc:51-64
    map2alm_iter         alm_healpix_tools.cc:73-85
    alm2map_spin         alm_healpix_tools.cc:350-365
    map2alm_spin         alm_healpix_tools.cc:123-144
    alm2map_pol          alm_healpix_tools.cc:375-395
    map2alm_pol          alm_healpix_tools.cc:190-217
    map2alm_pol_iter     alm_healpix_tools.cc:239-265
    alm2map_der1         alm_healpix_tools.cc:412-428

and the a_lm-side steps and module bodies of the programs built on them
(without their file I/O, which stays with the caller):

    scale_l              Healpix_cxx/alm.h:122-129 (Alm::ScaleL)
    smooth_with_gauss    Healpix_cxx/alm_powspec_tools.cc:250-283
    apply_cosine_window  Healpix_cxx/alm_powspec_tools.cc:285-299
    alm2map_cxx          Healpix_cxx/alm2map_cxx_module.cc:80-127
    anafast_cxx          Healpix_cxx/anafast_cxx_module.cc:55-127
    smoothing_cxx        Healpix_cxx/smoothing_cxx_module.cc:49-115

The Jacobi sweeps of map2alm_iter form their correction in a_lm space:
a <- a + a0 - YtW(Y a) with a0 = YtW(map), which equals the reference's
a <- a + YtW(map - Y a) up to rounding.  The subtraction runs inside the
analysis (SHARP_SUBTRACT), so no residual map is formed in a separate pass.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import (SHARP_ADD, SHARP_ALM2MAP, SHARP_ALM2MAP_DERIV1, SHARP_DP, SHARP_MAP2ALM,
               SHARP_SUBTRACT, AlmInfo, Geometry, execute_device)

FOURPI = 12.56637061435917295385057353311801153679      # cxxsupport/lsconstants.h:38
FWHM2SIGMA = 1.0 / 2.3548200450309493                   # lsconstants.h:56-57
HEALPIX_UNDEF = -1.6375e30                              # value of an undefined pixel

_GEOM: dict = {}
_ALM: dict = {}


def geometry(nside: int, weight=None) -> Geometry:
    """Cached HEALPix geometry (ring weights: 2*nside relative factors)."""
    key = (nside, None if weight is None else tuple(float(x) for x in weight))
    if key not in _GEOM:
        _GEOM[key] = Geometry.healpix(nside, weight)
    return _GEOM[key]


def alm_info(lmax: int, mmax: int | None = None) -> AlmInfo:
    key = (lmax, lmax if mmax is None else mmax)
    if key not in _ALM:
        _ALM[key] = AlmInfo.triangular(*key)
    return _ALM[key]


def _f64(t: torch.Tensor) -> torch.Tensor:
    """Real view of a complex128 tensor (the ABI takes interleaved re/im)."""
    if t.is_complex():
        return torch.view_as_real(t).reshape(-1)
    return t


def nside_of(map_: torch.Tensor) -> int:
    nside = int(round((map_.numel() / 12) ** 0.5))
    if 12 * nside * nside != map_.numel():
        raise ValueError("map size is not 12*nside^2")
    return nside


def alm2map(alm: torch.Tensor, map_: torch.Tensor, lmax: int, mmax: int | None = None,
            add: bool = False) -> torch.Tensor:
    nside = nside_of(map_)
    execute_device(SHARP_ALM2MAP, 0, [_f64(alm)], [map_], geometry(nside), alm_info(lmax, mmax),
                   1, SHARP_DP | (SHARP_ADD if add else 0))
    return map_


def map2alm(map_: torch.Tensor, alm: torch.Tensor, lmax: int, mmax: int | None = None,
            weight=None, add: bool = False) -> torch.Tensor:
    nside = nside_of(map_)
    execute_device(SHARP_MAP2ALM, 0, [_f64(alm)], [map_], geometry(nside, weight),
                   alm_info(lmax, mmax), 1, SHARP_DP | (SHARP_ADD if add else 0))
    return alm


def map2alm_iter(map_: torch.Tensor, alm: torch.Tensor, lmax: int, num_iter: int,
                 mmax: int | None = None, weight=None) -> torch.Tensor:
    """map2alm followed by num_iter Jacobi sweeps alm += map2alm(map - alm2map(alm))."""
    map2alm(map_, alm, lmax, mmax, weight)
    if num_iter <= 0:
        return alm
    nside = nside_of(map_)
    g, a = geometry(nside, weight), alm_info(lmax, mmax)
    a0 = alm.clone()
    work = torch.empty_like(map_)
    for _ in range(num_iter):
        alm2map(alm, work, lmax, mmax)
        alm.add_(a0)
        execute_device(SHARP_MAP2ALM, 0, [_f64(alm)], [work], g, a, 1,
                       SHARP_DP | SHARP_SUBTRACT)
    return alm


def alm2map_spin(alm1, alm2, map1, map2, spin: int, lmax: int, mmax: int | None = None,
                 add: bool = False):
    nside = nside_of(map1)
    execute_device(SHARP_ALM2MAP, spin, [_f64(alm1), _f64(alm2)], [map1, map2],
                   geometry(nside), alm_info(lmax, mmax), 1,
                   SHARP_DP | (SHARP_ADD if add else 0))
    return map1, map2


def map2alm_spin(map1, map2, alm1, alm2, spin: int, lmax: int, mmax: int | None = None,
                 weight=None, add: bool = False):
    nside = nside_of(map1)
    execute_device(SHARP_MAP2ALM, spin, [_f64(alm1), _f64(alm2)], [map1, map2],
                   geometry(nside, weight), alm_info(lmax, mmax), 1,
                   SHARP_DP | (SHARP_ADD if add else 0))
    return alm1, alm2


def alm2map_pol(almT, almG, almC, mapT, mapQ, mapU, lmax: int, mmax: int | None = None,
                add: bool = False):
    """T via spin 0, (Q, U) from (E, B) via spin 2."""
    alm2map(almT, mapT, lmax, mmax, add)
    alm2map_spin(almG, almC, mapQ, mapU, 2, lmax, mmax, add)
    return mapT, mapQ, mapU


def map2alm_pol(mapT, mapQ, mapU, almT, almG, almC, lmax: int, mmax: int | None = None,
                weight=None, add: bool = False):
    map2alm(mapT, almT, lmax, mmax, weight, add)
    map2alm_spin(mapQ, mapU, almG, almC, 2, lmax, mmax, weight, add)
    return almT, almG, almC


def map2alm_pol_iter(mapT, mapQ, mapU, almT, almG, almC, lmax: int, num_iter: int,
                     mmax: int | None = None, weight=None):
    map2alm_pol(mapT, mapQ, mapU, almT, almG, almC, lmax, mmax, weight)
    if num_iter <= 0:
        return almT, almG, almC
    nside = nside_of(mapT)
    g, a = geometry(nside, weight), alm_info(lmax, mmax)
    a0 = [x.clone() for x in (almT, almG, almC)]
    wT, wQ, wU = torch.empty_like(mapT), torch.empty_like(mapQ), torch.empty_like(mapU)
    for _ in range(num_iter):
        alm2map_pol(almT, almG, almC, wT, wQ, wU, lmax, mmax)
        for x, x0 in zip((almT, almG, almC), a0):
            x.add_(x0)
        execute_device(SHARP_MAP2ALM, 0, [_f64(almT)], [wT], g, a, 1, SHARP_DP | SHARP_SUBTRACT)
        execute_device(SHARP_MAP2ALM, 2, [_f64(almG), _f64(almC)], [wQ, wU], g, a, 1,
                       SHARP_DP | SHARP_SUBTRACT)
    return almT, almG, almC


def alm2map_der1(alm, map_, dth, dph, lmax: int, mmax: int | None = None):
    """Map and its first derivatives d/dtheta, d/dphi / sin(theta)."""
    alm2map(alm, map_, lmax, mmax)
    nside = nside_of(map_)
    execute_device(SHARP_ALM2MAP_DERIV1, 1, [_f64(alm)], [dth, dph], geometry(nside),
                   alm_info(lmax, mmax), 1, SHARP_DP)
    return map_, dth, dph


# ---------------------------------------------------------------------------
# a_lm-side steps of the Healpix_cxx programs
# ---------------------------------------------------------------------------
_LIDX: dict = {}


def l_index(lmax: int, mmax: int | None, device) -> torch.Tensor:
    """l of every entry of the triangular m-major layout (Alm<T> order)."""
    mmax = lmax if mmax is None else mmax
    key = (lmax, mmax, str(device))
    if key not in _LIDX:
        idx = np.concatenate([np.arange(m, lmax + 1) for m in range(mmax + 1)])
        _LIDX[key] = torch.from_numpy(idx).to(device)
    return _LIDX[key]


def scale_l(alm: torch.Tensor, factor, lmax: int, mmax: int | None = None) -> torch.Tensor:
    """alm(l, m) *= factor[l] for all l, m (Alm::ScaleL), in place on the device."""
    f = torch.as_tensor(np.asarray(factor, np.float64), device=alm.device)
    if f.numel() <= lmax:
        raise ValueError("alm.ScaleL: factor array too short")
    # real and imaginary parts times the real factor (no complex product)
    torch.view_as_real(alm).mul_(f[l_index(lmax, mmax, alm.device)].unsqueeze(-1))
    return alm


def gauss_beam(fwhm: float, lmax: int, pol: bool = False) -> np.ndarray:
    """exp(-l(l+1) sigma^2 / 2), sigma = fwhm / sqrt(8 ln 2) (fwhm in radians; a
    negative fwhm gives the inverse, a deconvolution); pol multiplies by
    exp(2 sigma^2) (the spin-2 beam of smoothWithGauss)."""
    fct = 1 if fwhm >= 0 else -1
    sigma = fwhm * FWHM2SIGMA
    l = np.arange(lmax + 1, dtype=np.float64)
    gb = np.exp(-.5 * fct * l * (l + 1) * sigma * sigma)
    if pol:
        gb = gb * math.exp(2 * fct * sigma * sigma)
    return gb


def smooth_with_gauss(alm: torch.Tensor, fwhm: float, lmax: int, mmax: int | None = None,
                      almG: torch.Tensor | None = None, almC: torch.Tensor | None = None):
    """Gaussian beam on T (and, if given, on the E/B pair with the spin-2
    factor), in place."""
    scale_l(alm, gauss_beam(fwhm, lmax), lmax, mmax)
    if almG is not None:
        gp = gauss_beam(fwhm, lmax, pol=True)
        scale_l(almG, gp, lmax, mmax)
        scale_l(almC, gp, lmax, mmax)
    return alm


def cosine_window(lmin: int, lmax_w: int, lmax: int) -> np.ndarray:
    """1 below lmin, (1 + cos(pi (l - lmin)/(lmax_w - lmin)))/2 up to lmax_w, 0 above."""
    if not (lmin >= 0 and lmax_w > lmin):
        raise ValueError("bad lmin/lmax")
    cw = np.zeros(lmax + 1)
    for i in range(lmax + 1):
        if i < lmin:
            cw[i] = 1.0
        elif i < lmax_w:
            cw[i] = (1 + math.cos(math.pi * (i - lmin) / float(lmax_w - lmin))) / 2
    return cw


def apply_cosine_window(alm: torch.Tensor, lmin: int, lmax_w: int, lmax: int,
                        mmax: int | None = None) -> torch.Tensor:
    return scale_l(alm, cosine_window(lmin, lmax_w, lmax), lmax, mmax)


def _defined(map_: torch.Tensor) -> torch.Tensor:
    """Pixels that are not the undefined value (relative tolerance 1e-5)."""
    return (map_ - HEALPIX_UNDEF).abs() > 1e-5 * abs(HEALPIX_UNDEF)


def _monopole_out(map_: torch.Tensor):
    """Average of the defined pixels, subtracted from them; undefined pixels
    set to 0.  Returns the average as a 0-dim device tensor."""
    ok = _defined(map_)
    avg = map_[ok].sum() / ok.sum()
    map_.sub_(torch.where(ok, avg, torch.zeros_like(avg)))
    map_.masked_fill_(~ok, 0.0)
    return avg


def alm2map_cxx(alm, map_, lmax: int, mmax: int | None = None, fwhm: float = 0.0,
                pixwin=None, cosine=None, almG=None, almC=None, mapQ=None, mapU=None,
                pixwin_pol=None):
    """Body of alm2map_cxx on device tensors: beam (fwhm in radians, applied
    when > 0), optional cosine window (lmin, lmax), pixel window, then the
    map with the monopole a_00 added as a constant offset.  With almG/almC
    and mapQ/mapU the polarised branch runs (pixwin_pol on E/B).  The input
    a_lm are not modified."""
    pol = almG is not None
    a = alm.clone()
    g = almG.clone() if pol else None
    c = almC.clone() if pol else None
    if fwhm > 0:
        smooth_with_gauss(a, fwhm, lmax, mmax, g, c)
    if cosine is not None:
        for x in (a, g, c):
            if x is not None:
                apply_cosine_window(x, cosine[0], cosine[1], lmax, mmax)
    if pixwin is not None:
        scale_l(a, pixwin, lmax, mmax)
    if pol and pixwin_pol is not None:
        scale_l(g, pixwin_pol, lmax, mmax)
        scale_l(c, pixwin_pol, lmax, mmax)
    offset = a[0].real / math.sqrt(FOURPI)
    a[0] = 0
    if pol:
        alm2map_pol(a, g, c, map_, mapQ, mapU, lmax, mmax)
    else:
        alm2map(a, map_, lmax, mmax)
    map_.add_(offset)
    return (map_, mapQ, mapU) if pol else map_


def anafast_cxx(map_, alm, lmax: int, num_iter: int = 0, mmax: int | None = None,
                weight=None, remove_monopole: bool = False, mapQ=None, mapU=None, almG=None,
                almC=None):
    """Body of anafast_cxx up to the a_lm (the power spectrum is
    extract_powspec of the result): optional monopole removal, undefined
    pixels set to 0, map2alm_iter (map2alm_pol_iter with Q/U), the monopole
    restored in a_00.  The input maps are not modified."""
    pol = mapQ is not None
    t = map_.clone()
    avg = _monopole_out(t) if remove_monopole else None
    if not remove_monopole:
        t.masked_fill_(~_defined(t), 0.0)
    if pol:
        q, u = mapQ.clone(), mapU.clone()
        for x in (q, u):
            x.masked_fill_(~_defined(x), 0.0)
        map2alm_pol_iter(t, q, u, alm, almG, almC, lmax, num_iter, mmax, weight)
    else:
        map2alm_iter(t, alm, lmax, num_iter, mmax, weight)
    if avg is not None:
        alm[0] += avg * math.sqrt(FOURPI)
    return (alm, almG, almC) if pol else alm


def smoothing_cxx(map_, lmax: int, fwhm: float, num_iter: int = 0, weight=None, mapQ=None,
                  mapU=None):
    """Body of smoothing_cxx in place on device maps: monopole out, analysis
    with num_iter Jacobi sweeps, Gaussian beam (fwhm in radians; negative
    deconvolves), synthesis, monopole back.  lmax = mmax as there."""
    pol = mapQ is not None
    avg = _monopole_out(map_)
    n = (lmax + 1) * (lmax + 2) // 2
    mk = lambda: torch.zeros(n, dtype=torch.complex128, device=map_.device)  # noqa: E731
    a = mk()
    if pol:
        for x in (mapQ, mapU):
            x.masked_fill_(~_defined(x), 0.0)
        g, c = mk(), mk()
        map2alm_pol_iter(map_, mapQ, mapU, a, g, c, lmax, num_iter, None, weight)
        smooth_with_gauss(a, fwhm, lmax, None, g, c)
        alm2map_pol(a, g, c, map_, mapQ, mapU, lmax)
    else:
        map2alm_iter(map_, a, lmax, num_iter, None, weight)
        smooth_with_gauss(a, fwhm, lmax)
        alm2map(a, map_, lmax)
    map_.add_(avg)
    return (map_, mapQ, mapU) if pol else map_
