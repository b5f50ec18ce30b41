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
"""
from __future__ import annotations

import torch

from . import (SHARP_ADD, SHARP_ALM2MAP, SHARP_ALM2MAP_DERIV1, SHARP_DP, SHARP_MAP2ALM,
               AlmInfo, Geometry, execute_device)

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
    work = torch.empty_like(map_)
    for _ in range(num_iter):
        alm2map(alm, work, lmax, mmax)
        torch.sub(map_, work, out=work)
        map2alm(work, alm, lmax, mmax, weight, add=True)
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
    wT, wQ, wU = torch.empty_like(mapT), torch.empty_like(mapQ), torch.empty_like(mapU)
    for _ in range(num_iter):
        alm2map_pol(almT, almG, almC, wT, wQ, wU, lmax, mmax)
        torch.sub(mapT, wT, out=wT)
        torch.sub(mapQ, wQ, out=wQ)
        torch.sub(mapU, wU, out=wU)
        map2alm_pol(wT, wQ, wU, almT, almG, almC, lmax, mmax, weight, add=True)
    return almT, almG, almC


def alm2map_der1(alm, map_, dth, dph, lmax: int, mmax: int | None = None):
    """Map and its first derivatives d/dtheta, d/dphi / sin(theta)."""
    alm2map(alm, map_, lmax, mmax)
    nside = nside_of(map_)
    execute_device(SHARP_ALM2MAP_DERIV1, 1, [_f64(alm)], [dth, dph], geometry(nside),
                   alm_info(lmax, mmax), 1, SHARP_DP)
    return map_, dth, dph
