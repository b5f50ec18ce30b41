"""Differentiable spherical-harmonic transforms for torch.

The backward passes call the library's adjoint transforms (the SHARP_ADJOINT
flag of sharp_b200.h), not autograd of a reimplementation:

* alm2map  m = Y a.  Y is real-linear in x = (Re a, Im a).  The library's Yt
  satisfies <Y a, m> = sum_{m=0} Re(a* Yt m) + 2 sum_{m>0} Re(a* Yt m), so
  dL/dx = D Yt(dL/dm) with D = 1 on the m=0 block and 2 elsewhere; Im a_l0 is
  not an input of Y and receives zero gradient.
* map2alm  a = Yt W m.  Its plain transpose is W Y D^-1, so
  dL/dm = W Y (D^-1 dL/dx): the adjoint of map2alm is the weighted synthesis.

Tensors: a_lm complex128 (triangular m-major layout, one tensor per
component), maps float64, all on the same CUDA device.

precision="mixed" runs the forward transform and its adjoint with
SHARP_MIXED (the int8 tensor-core Legendre step, within 1e-6 relative L2 of
FP64); precision="fp64" (default) runs both in FP64.
"""
from __future__ import annotations

import torch

from . import (SHARP_ADJOINT, SHARP_ALM2MAP, SHARP_DP, SHARP_MAP2ALM, SHARP_MIXED, AlmInfo,
               Geometry, execute_device)

_PRECISION = {"fp64": SHARP_DP, "mixed": SHARP_DP | SHARP_MIXED}


def _flags(precision: str) -> int:
    try:
        return _PRECISION[precision]
    except KeyError:
        raise ValueError(f"precision must be one of {sorted(_PRECISION)}") from None


def _real(t: torch.Tensor) -> torch.Tensor:
    return torch.view_as_real(t).reshape(-1)


def _m_weights(lmax: int, mmax: int, device) -> torch.Tensor:
    """D: 1 on the m = 0 block (first lmax+1 entries), 2 elsewhere."""
    nalm = ((mmax + 1) * (mmax + 2)) // 2 + (mmax + 1) * (lmax - mmax)
    w = torch.full((nalm,), 2.0, dtype=torch.float64, device=device)
    w[: lmax + 1] = 1.0
    return w


class _Alm2Map(torch.autograd.Function):
    @staticmethod
    def forward(ctx, geom: Geometry, ainfo: AlmInfo, spin: int, npix: int, flags: int, *alms):
        ctx.geom, ctx.ainfo, ctx.spin, ctx.flags = geom, ainfo, spin, flags
        maps = [torch.empty(npix, dtype=torch.float64, device=alms[0].device)
                for _ in alms]
        alm_in = [a.detach().contiguous() for a in alms]  # Im a_l0 is ignored by Y
        execute_device(SHARP_ALM2MAP, spin, [_real(a) for a in alm_in], maps, geom, ainfo, 1,
                       flags)
        return tuple(maps) if len(maps) > 1 else maps[0]

    @staticmethod
    def backward(ctx, *gmaps):
        geom, ainfo, spin = ctx.geom, ctx.ainfo, ctx.spin
        lmax, nm = ainfo.lmax, ainfo.nm
        gm = [g.contiguous() for g in gmaps]
        galm = [torch.zeros(ainfo.nalm(), dtype=torch.complex128, device=gm[0].device)
                for _ in gm]
        # Yt through the adjoint flag on the synthesis job type
        execute_device(SHARP_ALM2MAP, spin, [_real(a) for a in galm], gm, geom, ainfo, 1,
                       ctx.flags | SHARP_ADJOINT)
        w = _m_weights(lmax, nm - 1, gm[0].device)
        galm = [a * w for a in galm]
        return (None, None, None, None, None, *galm)


class _Map2Alm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, geom: Geometry, ainfo: AlmInfo, spin: int, flags: int, *maps):
        ctx.geom, ctx.ainfo, ctx.spin, ctx.flags = geom, ainfo, spin, flags
        alms = [torch.zeros(ainfo.nalm(), dtype=torch.complex128, device=maps[0].device)
                for _ in maps]
        execute_device(SHARP_MAP2ALM, spin, [_real(a) for a in alms],
                       [m.detach().contiguous() for m in maps], geom, ainfo, 1, flags)
        return tuple(alms) if len(alms) > 1 else alms[0]

    @staticmethod
    def backward(ctx, *galms):
        geom, ainfo, spin = ctx.geom, ctx.ainfo, ctx.spin
        lmax, nm = ainfo.lmax, ainfo.nm
        w = _m_weights(lmax, nm - 1, galms[0].device)
        ga = [(g.contiguous() / w) for g in galms]
        npix = geom.npix()
        gmaps = [torch.zeros(npix, dtype=torch.float64, device=ga[0].device) for _ in ga]
        # (Yt W)^T = W Y: the adjoint of the analysis job type
        execute_device(SHARP_MAP2ALM, spin, [_real(a) for a in ga], gmaps, geom, ainfo, 1,
                       ctx.flags | SHARP_ADJOINT)
        return (None, None, None, None, *gmaps)


def alm2map(geom: Geometry, ainfo: AlmInfo, spin: int, *alms: torch.Tensor,
            precision: str = "fp64"):
    """Differentiable synthesis: spin 0 takes one a_lm tensor, spin > 0 two
    (E, B); returns one map or a (Q, U) tuple."""
    return _Alm2Map.apply(geom, ainfo, spin, geom.npix(), _flags(precision), *alms)


def map2alm(geom: Geometry, ainfo: AlmInfo, spin: int, *maps: torch.Tensor,
            precision: str = "fp64"):
    """Differentiable analysis (with the geometry's quadrature weights)."""
    return _Map2Alm.apply(geom, ainfo, spin, _flags(precision), *maps)
