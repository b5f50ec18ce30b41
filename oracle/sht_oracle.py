"""CPU oracle: a numpy restatement of libsharp's ``sharp_execute`` path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use it, always as the checker.  It is written for clarity at small sizes
(lmax up to a few hundred): Python loops over m and l, numpy over rings.

Parity is pinned two ways (see tests/test_oracle.py):
  * against the 18 hard-coded golden values of the reference test suite
    (libsharp/sharp_testsuite.c:376-434, ``check_sign_scale``), and
  * against the reference libsharp compiled from its own sources
    (oracle/Makefile -> oracle/_ref/libsharp_ref.so), on seeded inputs.

Each function names the reference file:line it restates.  Paths are relative
to the zonca/planck-levelS source tree.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Flags and job types (libsharp/sharp_lowlevel.h:160-191)
# ---------------------------------------------------------------------------
SHARP_MAP2ALM = 0
SHARP_ALM2MAP = 1
SHARP_Yt = 2
SHARP_WY = 3
SHARP_ALM2MAP_DERIV1 = 4
SHARP_DP = 1 << 4
SHARP_ADD = 1 << 5
SHARP_REAL_HARMONICS = 1 << 6
SHARP_NO_FFT = 1 << 7
SHARP_USE_WEIGHTS = 1 << 20
SHARP_PACKED = 1  # alm_info flag, sharp_lowlevel.h:89

# scale constants, libsharp/sharp_ylmgen_c.h:39-42
FBIG = 2.0 ** 800
FSMALL = 2.0 ** -800
FTOL = 2.0 ** -60
FBIGHALF = 2.0 ** 400
MINSCALE, LIMSCALE = 0, 1
SQRT_ONE_HALF = math.sqrt(0.5)
SQRT_TWO = math.sqrt(2.0)


# ---------------------------------------------------------------------------
# Geometry (libsharp/sharp.c:122-135, 179-227; sharp_geomhelpers.c)
# ---------------------------------------------------------------------------
@dataclass
class Ring:
    theta: float
    phi0: float
    weight: float
    cth: float
    sth: float
    ofs: int
    nph: int
    stride: int


@dataclass
class Geometry:
    pairs: list = field(default_factory=list)  # list of (Ring, Ring|None)
    nphmax: int = 0


def make_geom_info(nph, ofs, stride, phi0, theta, wgt=None) -> Geometry:
    """sharp_make_geom_info, libsharp/sharp.c:179-227: sort rings by sin(theta),
    pair rings with cth ~ -cth (rel. 1e-12, north ring first), then sort pairs
    by (nph, phi0, cth descending)."""
    n = len(nph)
    rings = []
    for i in range(n):
        th = float(theta[i])
        rings.append(Ring(th, float(phi0[i]), 1.0 if wgt is None else float(wgt[i]),
                          math.cos(th), math.sin(th), int(ofs[i]), int(nph[i]),
                          int(stride[i])))
    rings.sort(key=lambda r: r.sth)  # qsort on sth (ties: order irrelevant)
    geo = Geometry(nphmax=max(int(x) for x in nph))
    pos = 0
    while pos < n:
        r1, r2 = rings[pos], None
        if pos < n - 1 and _fapprox(rings[pos].cth, -rings[pos + 1].cth, 1e-12):
            if rings[pos].cth > 0:
                r2 = rings[pos + 1]
            else:
                r1, r2 = rings[pos + 1], rings[pos]
            pos += 1
        geo.pairs.append((r1, r2))
        pos += 1
    geo.pairs.sort(key=lambda p: (p[0].nph, p[0].phi0, -p[0].cth))
    return geo


def _fapprox(a, b, eps):
    # c_utils/c_utils.h:124-125 FAPPROX: fabs(a-b) < eps*fabs(b)
    return abs(a - b) < eps * abs(b)


def healpix_geometry(nside: int, weight=None, stride: int = 1) -> Geometry:
    """sharp_make_weighted_healpix_geom_info, libsharp/sharp_geomhelpers.c:38-93."""
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    nrings = 4 * nside - 1
    theta = np.zeros(nrings); nph = np.zeros(nrings, np.int64)
    phi0 = np.zeros(nrings); ofs = np.zeros(nrings, np.int64)
    wgt = np.zeros(nrings)
    for m in range(nrings):
        ring = m + 1
        northring = 4 * nside - ring if ring > 2 * nside else ring
        if northring < nside:
            theta[m] = 2 * math.asin(northring / (math.sqrt(6.0) * nside))
            nph[m] = 4 * northring
            phi0[m] = math.pi / nph[m]
            ofs[m] = 2 * northring * (northring - 1) * stride
        else:
            fact1 = (8.0 * nside) / npix
            costheta = (2 * nside - northring) * fact1
            theta[m] = math.acos(costheta)
            nph[m] = 4 * nside
            phi0[m] = 0.0 if ((northring - nside) & 1) else math.pi / nph[m]
            ofs[m] = (ncap + (northring - nside) * nph[m]) * stride
        if northring != ring:
            theta[m] = math.pi - theta[m]
            ofs[m] = (npix - nph[m]) * stride - ofs[m]
        wgt[m] = 4.0 * math.pi / npix * (1.0 if weight is None else weight[northring - 1])
    return make_geom_info(nph, ofs, np.full(nrings, stride), phi0, theta, wgt)


def gauss_legendre_nodes(n: int):
    """Gauss-Legendre nodes/weights by Newton iteration on P_n (the reference
    uses the same method, libsharp/sharp_geomhelpers.c:105-156).  Returns x
    ascending and weights."""
    x = np.zeros(n); w = np.zeros(n)
    for i in range(1, (n + 1) // 2 + 1):
        x0 = math.cos(math.pi * (4 * i - 1) / (4 * n + 2)) * (1 - (1 - 1.0 / n) / (8.0 * n * n))
        for it in range(100):
            p1, p0 = 1.0, x0
            for k in range(2, n + 1):
                p2, p1 = p1, p0
                p0 = x0 * p1 + (k - 1.0) / k * (x0 * p1 - p2)
            omx2 = (1 + x0) * (1 - x0) if abs(x0) > 0.1 else 1 - x0 * x0
            dpdx = (p1 - x0 * p0) * n / omx2
            dx = p0 / dpdx
            x0 -= dx
            if abs(dx) <= 1e-16 * max(1.0, abs(x0)) and it > 1:
                break
        p1, p0 = 1.0, x0
        for k in range(2, n + 1):
            p2, p1 = p1, p0
            p0 = x0 * p1 + (k - 1.0) / k * (x0 * p1 - p2)
        omx2 = (1 + x0) * (1 - x0) if abs(x0) > 0.1 else 1 - x0 * x0
        dpdx = (p1 - x0 * p0) * n / omx2
        x[i - 1] = -x0; x[n - i] = x0
        w[i - 1] = w[n - i] = 2.0 / (omx2 * dpdx * dpdx)
    return x, w


def gauss_geometry(nrings: int, nphi: int, phi0: float = 0.0,
                   stride_lon: int = 1, stride_lat: int | None = None) -> Geometry:
    """sharp_make_gauss_geom_info, libsharp/sharp_geomhelpers.c:158-190."""
    if stride_lat is None:
        stride_lat = nphi
    x, w = gauss_legendre_nodes(nrings)
    theta = np.arccos(-x)
    wgt = w * 2 * math.pi / nphi
    return make_geom_info(np.full(nrings, nphi), np.arange(nrings) * stride_lat,
                          np.full(nrings, stride_lon), np.full(nrings, phi0), theta, wgt)


# ---------------------------------------------------------------------------
# a_lm layout (libsharp/sharp_almhelpers.c:35-52)
# ---------------------------------------------------------------------------
@dataclass
class AlmInfo:
    lmax: int
    mval: np.ndarray
    mvstart: np.ndarray
    stride: int = 1
    flags: int = 0

    @property
    def nm(self):
        return len(self.mval)


def triangular_alm_info(lmax: int, mmax: int, stride: int = 1) -> AlmInfo:
    m = np.arange(mmax + 1, dtype=np.int64)
    return AlmInfo(lmax, m.astype(np.int32), stride * ((m * (2 * lmax + 1 - m)) >> 1), stride)


def nalm_triangular(lmax, mmax):
    return ((mmax + 1) * (mmax + 2)) // 2 + (mmax + 1) * (lmax - mmax)


# ---------------------------------------------------------------------------
# Recurrence coefficients (libsharp/sharp_ylmgen_c.c)
# ---------------------------------------------------------------------------
def _normalize(val, scale, xfmax):
    # sharp_ylmgen_c.c:37-42
    while abs(val) > xfmax:
        val *= FSMALL; scale += 1
    if val != 0.0:
        while abs(val) < xfmax * FSMALL:
            val *= FBIG; scale -= 1
    return val, scale


class Ylmgen:
    """sharp_Ylmgen_init / _prepare (libsharp/sharp_ylmgen_c.c:44-198)."""

    def __init__(self, lmax, mmax, spin):
        self.lmax, self.mmax, self.s = lmax, mmax, spin
        if spin == 0:
            root = np.sqrt(np.arange(2 * lmax + 5, dtype=np.float64))
            iroot = np.zeros_like(root); iroot[1:] = 1.0 / root[1:]
            self.root, self.iroot = root, iroot
            mfac = np.zeros(mmax + 1); mfac[0] = 0.2820947917738781434740397257803862929220
            for m in range(1, mmax + 1):
                mfac[m] = mfac[m - 1] * math.sqrt((2 * m + 1.0) / (2 * m))
            self.mfac = mfac
        else:
            self.inv = np.zeros(lmax + 1); self.inv[1:] = 1.0 / np.arange(1, lmax + 1)
            k = np.arange(2 * lmax + 1, dtype=np.float64)
            self.flm1 = np.sqrt(1.0 / (k + 1.0))
            self.flm2 = np.sqrt(k / (k + 1.0))
            fac = [1.0]; facscale = [0]
            for m in range(1, 2 * lmax + 1):
                v, s = _normalize(fac[-1] * math.sqrt(m), facscale[-1], FBIGHALF)
                fac.append(v); facscale.append(s)
            self.prefac = np.zeros(mmax + 1); self.fscale = np.zeros(mmax + 1, np.int64)
            for m in range(mmax + 1):
                mlo, mhi = sorted((spin, m))
                tfac = fac[2 * mhi] / fac[mhi + mlo]
                tscale = facscale[2 * mhi] - facscale[mhi + mlo]
                tfac, tscale = _normalize(tfac, tscale, FBIGHALF)
                tfac /= fac[mhi - mlo]
                tscale -= facscale[mhi - mlo]
                tfac, tscale = _normalize(tfac, tscale, FBIGHALF)
                self.prefac[m] = tfac; self.fscale[m] = tscale

    def prepare(self, m):
        lmax, s = self.lmax, self.s
        self.m = m
        if s == 0:
            rf = np.zeros((lmax + 1, 2))
            rf[m, 0] = self.root[2 * m + 3]
            l = np.arange(m + 1, lmax + 1)
            tmp = self.root[2 * l + 3] * self.iroot[l + 1 + m] * self.iroot[l + 1 - m]
            rf[l, 0] = tmp * self.root[2 * l + 1]
            rf[l, 1] = tmp * self.root[l + m] * self.root[l - m] * self.iroot[2 * l - 1]
            self.rf = rf
        else:
            mlo, mhi = sorted((m, s))
            self.mlo, self.mhi = mlo, mhi
            fx = np.zeros((lmax + 2, 3))
            l = np.arange(mhi, lmax)
            t = self.flm1[l + m] * self.flm1[l - m] * self.flm1[l + s] * self.flm1[l - s]
            fx[l + 1, 0] = (l + 1.0) * (2 * l + 1.0) * t
            fx[l + 1, 1] = m * s * self.inv[l] * self.inv[l + 1]
            t = self.flm2[l + m] * self.flm2[l - m] * self.flm2[l + s] * self.flm2[l - s]
            fx[l + 1, 2] = t * (l + 1.0) * self.inv[l]
            self.fx = fx
            if mhi == m:
                self.cosPow, self.sinPow = mhi + s, mhi - s
                self.preMinus_p = self.preMinus_m = (mhi - s) & 1
            else:
                self.cosPow, self.sinPow = mhi + m, mhi - m
                self.preMinus_p, self.preMinus_m = 0, (mhi + m) & 1


def get_norm(lmax, spin):
    """sharp_Ylmgen_get_norm, libsharp/sharp_ylmgen_c.c:200-222."""
    if spin == 0:
        return np.ones(lmax + 1)
    spinsign = -1.0 if spin > 0 else 1.0
    if spin & 1:
        spinsign = -spinsign
    l = np.arange(lmax + 1)
    return np.where(l < spin, 0.0, spinsign * 0.5 * np.sqrt((2 * l + 1) / (4 * math.pi)))


def get_d1norm(lmax):
    """sharp_Ylmgen_get_d1norm, libsharp/sharp_ylmgen_c.c:224-232."""
    l = np.arange(lmax + 1, dtype=np.float64)
    return np.where(l < 1, 0.0, 0.5 * np.sqrt(l * (l + 1) * (2 * l + 1) / (4 * math.pi)))


def get_mlim(lmax, spin, sth, cth):
    """sharp_get_mlim, libsharp/sharp.c:66-78."""
    ofs = max(lmax * 0.01, 100.0)
    b = -2 * spin * abs(cth)
    t1 = lmax * sth + ofs
    c = float(spin) * spin - t1 * t1
    discr = b * b - 4 * c
    if discr <= 0:
        return lmax
    res = (-b + math.sqrt(discr)) / 2.0
    return int(min(res, lmax) + 0.5)


# ---------------------------------------------------------------------------
# Scaled arithmetic, vectorised over rings (libsharp/sharp_core_inc.c:73-207)
# ---------------------------------------------------------------------------
def _vnormalize(val, scale, maxval):
    # Tbnormalize, sharp_core_inc.c:73-95 (per ring)
    val = val.copy(); scale = scale.copy()
    while True:
        big = np.abs(val) > maxval
        if not big.any():
            break
        val[big] *= FSMALL; scale[big] += 1
    while True:
        small = (np.abs(val) < FSMALL * maxval) & (val != 0)
        if not small.any():
            break
        val[small] *= FBIG; scale[small] -= 1
    return val, scale


def _vpow(base, npow):
    # mypow, sharp_core_inc.c:97-126
    scale = np.zeros(base.shape, np.int64); scaleint = np.zeros(base.shape, np.int64)
    res = np.ones_like(base)
    val, scaleint = _vnormalize(base, scaleint, FBIGHALF)
    while True:
        if npow & 1:
            res = res * val; scale = scale + scaleint
            res, scale = _vnormalize(res, scale, FBIGHALF)
        val = val * val; scaleint = scaleint + scaleint
        val, scaleint = _vnormalize(val, scaleint, FBIGHALF)
        npow >>= 1
        if npow == 0:
            break
    return res, scale


def _corfac(scale):
    # getCorfac, sharp_core_inc.c:171-180 (cf[0]=1, cf[1]=2^800)
    out = np.zeros(scale.shape)
    out[scale == 0] = 1.0
    out[scale == 1] = FBIG
    return out


def legendre_spin0(gen: Ylmgen, m, cth, sth):
    """lambda_lm(theta) for l=m..lmax at fixed m, one column per ring.

    Restates iter_to_ieee + calc_alm2map (sharp_core_inc.c:182-207,
    sharp_core_inc2.c:164-220): scaled recurrence until the value is IEEE
    representable, contributions with scale<0 are exactly 0.  Vectorised per
    ring (the reference couples rings of one SIMD block; that only changes
    contributions below 2^-60 of the leading terms)."""
    lmax = gen.lmax
    rf = gen.rf
    nr = len(cth)
    out = np.zeros((lmax + 1, nr))
    lam2, scale = _vpow(sth, m)
    lam2 = lam2 * (-gen.mfac[m] if (m & 1) else gen.mfac[m])
    lam2, scale = _vnormalize(lam2, scale, FTOL)
    lam1 = np.zeros(nr)
    l = m
    out[l] = lam2 * _corfac(scale)
    while l < lmax:
        # lam_{l+1} = cth*lam_l*rf[l].f0 - lam_{l-1}*rf[l].f1
        lamn = cth * lam2 * rf[l, 0] - lam1 * rf[l, 1]
        lam1, lam2 = lam2, lamn
        l += 1
        # rescale (sharp_core_inc.c:128-144): keep magnitude <= ftol while scaled
        scaled = scale < LIMSCALE
        big = scaled & (np.abs(lam2) > FTOL)
        if big.any():
            lam1[big] *= FSMALL; lam2[big] *= FSMALL; scale[big] += 1
        out[l] = lam2 * _corfac(scale)
    return out


def legendre_spin(gen: Ylmgen, m, cth, sth):
    """(r+, r-) for l=mhi..lmax at fixed m (rows below mhi are zero).

    Restates iter_to_ieee_spin / calc_alm2map_spin (sharp_core_inc.c:223-293,
    sharp_core_inc2.c:432-476)."""
    lmax, s = gen.lmax, gen.s
    fx = gen.fx
    nr = len(cth)
    cth2 = np.maximum(np.sqrt((1.0 + cth) * 0.5), 1e-15)
    sth2 = np.maximum(np.sqrt((1.0 - cth) * 0.5), 1e-15)
    neg = sth < 0
    cth2 = np.where(neg & (cth < 0), -cth2, cth2)
    sth2 = np.where(neg & (cth > 0), -sth2, sth2)
    ccp, ccps = _vpow(cth2, gen.cosPow)
    ssp, ssps = _vpow(sth2, gen.sinPow)
    csp, csps = _vpow(cth2, gen.sinPow)
    scp, scps = _vpow(sth2, gen.cosPow)
    rec2p = gen.prefac[m] * ccp; scalep = gen.fscale[m] + ccps
    rec2m = gen.prefac[m] * csp; scalem = gen.fscale[m] + csps
    rec2m, scalem = _vnormalize(rec2m, scalem, FBIGHALF)
    rec2p, scalep = _vnormalize(rec2p, scalep, FBIGHALF)
    rec2p = rec2p * ssp; scalep = scalep + ssps
    rec2m = rec2m * scp; scalem = scalem + scps
    if gen.preMinus_p:
        rec2p = -rec2p
    if gen.preMinus_m:
        rec2m = -rec2m
    if s & 1:
        rec2p = -rec2p
    rec2m, scalem = _vnormalize(rec2m, scalem, FTOL)
    rec2p, scalep = _vnormalize(rec2p, scalep, FTOL)
    rec1p = np.zeros(nr); rec1m = np.zeros(nr)
    outp = np.zeros((lmax + 1, nr)); outm = np.zeros((lmax + 1, nr))
    l = gen.mhi
    outp[l] = rec2p * _corfac(scalep); outm[l] = rec2m * _corfac(scalem)
    while l < lmax:
        f0, f1, f2 = fx[l + 1]
        np_ = (cth - f1) * (f0 * rec2p) - f2 * rec1p
        nm_ = (cth + f1) * (f0 * rec2m) - f2 * rec1m
        rec1p, rec2p = rec2p, np_
        rec1m, rec2m = rec2m, nm_
        l += 1
        for (r1, r2, sc) in ((rec1p, rec2p, scalep), (rec1m, rec2m, scalem)):
            big = (sc < LIMSCALE) & (np.abs(r2) > FTOL)
            if big.any():
                r1[big] *= FSMALL; r2[big] *= FSMALL; sc[big] += 1
        outp[l] = rec2p * _corfac(scalep); outm[l] = rec2m * _corfac(scalem)
    return outp, outm


# ---------------------------------------------------------------------------
# Ring <-> phase (libsharp/sharp.c:253-353)
# ---------------------------------------------------------------------------
def phase2ring(ring: Ring, phase, mmax, flags):
    """ringhelper_phase2ring, libsharp/sharp.c:253-303, including the alias
    fold for nph < 2*mmax+1 and FFTPACK's backward real transform (unnormalised,
    imaginary parts of bins 0 and nph/2 dropped)."""
    nph = ring.nph
    wgt = ring.weight if (flags & SHARP_USE_WEIGHTS) else 1.0
    if flags & SHARP_REAL_HARMONICS:
        wgt *= SQRT_ONE_HALF
    m = np.arange(mmax + 1)
    tmp = phase[: mmax + 1] * wgt
    if abs(ring.phi0) >= 1e-14:
        tmp = tmp * np.exp(1j * m * ring.phi0)
    half = nph // 2 + 1
    spec = np.zeros(half, np.complex128)
    spec[0] += tmp[0].real
    if mmax >= 1:
        mm = m[1:]; t = tmp[1:]
        # the reference's running index starts at 1 for m = 1 and wraps only
        # after it (sharp.c:282, :297): for a one-pixel ring the direct term
        # of m = 1 falls outside the bins and is dropped
        i1 = np.where(mm == 1, 1, mm % nph)
        ok1 = i1 < (nph + 2) // 2
        np.add.at(spec, i1[ok1], t[ok1])
        i2 = (nph - mm % nph) % nph
        ok2 = i2 < (nph + 2) // 2
        np.add.at(spec, i2[ok2], np.conj(t[ok2]))
    spec[0] = spec[0].real
    if nph % 2 == 0:
        spec[nph // 2] = spec[nph // 2].real
    # x_j = sum_k C_k e^{+2 pi i jk/n}, hermitian C: numpy irfft * n
    return np.fft.irfft(spec, n=nph) * nph


def ring2phase(ring: Ring, data, mmax, flags):
    """ringhelper_ring2phase, libsharp/sharp.c:305-353 (maxidx = mmax)."""
    nph = ring.nph
    wgt = ring.weight if (flags & SHARP_USE_WEIGHTS) else 1.0
    if flags & SHARP_REAL_HARMONICS:
        wgt *= SQRT_TWO
    full = np.fft.fft(data)  # D_k = sum_j x_j e^{-2 pi i jk/n}
    full[0] = full[0].real
    if nph % 2 == 0:
        full[nph // 2] = full[nph // 2].real
    m = np.arange(mmax + 1)
    val = full[m % nph] * wgt
    if abs(ring.phi0) >= 1e-14:
        val = val * np.exp(-1j * m * ring.phi0)
    return val


# ---------------------------------------------------------------------------
# Job driver (libsharp/sharp.c:408-629, 762-880; sharp_core_inc2.c:624-801)
# ---------------------------------------------------------------------------
def execute(jtype, spin, alm, maps, geom: Geometry, ainfo: AlmInfo, ntrans, flags):
    """Restates sharp_execute (double precision, host arrays).

    ``alm``: list of ntrans*nalm complex128 arrays (reference layout via
    ainfo).  ``maps``: list of ntrans*nmaps float64 arrays (complex128 with
    SHARP_NO_FFT).  Outputs are written in place (overwritten unless SHARP_ADD).
    """
    if not (0 < ntrans <= 100):
        raise ValueError("bad number of simultaneous transforms")
    if jtype == SHARP_ALM2MAP_DERIV1:
        spin = 1
    if jtype == SHARP_MAP2ALM:
        flags |= SHARP_USE_WEIGHTS
    if jtype == SHARP_Yt:
        jtype = SHARP_MAP2ALM
    if jtype == SHARP_WY:
        jtype = SHARP_ALM2MAP; flags |= SHARP_USE_WEIGHTS
    if not (0 <= spin <= ainfo.lmax):
        raise ValueError("bad spin")
    deriv = jtype == SHARP_ALM2MAP_DERIV1
    nmaps = 2 if (deriv or spin > 0) else 1
    nalm = 1 if deriv else (2 if spin > 0 else 1)
    lmax = ainfo.lmax
    mval = np.asarray(ainfo.mval)
    nm = len(mval)
    if sorted(mval.tolist()) != list(range(nm)):
        raise ValueError("not all m values are present")
    mmax = nm - 1
    norm_l = get_d1norm(lmax) if deriv else get_norm(lmax, spin)
    analysis = jtype == SHARP_MAP2ALM
    packed = bool(ainfo.flags & SHARP_PACKED)

    # init_output, sharp.c:444-453
    if not (flags & SHARP_ADD):
        if analysis:
            for a in alm:
                _alm_clear(a, ainfo)
        else:
            for mp in maps:
                for (r1, r2) in geom.pairs:
                    for r in (r1, r2):
                        if r is not None and r.nph > 0:
                            mp[r.ofs + np.arange(r.nph) * r.stride] = 0
    npairs = len(geom.pairs)
    ncomp = ntrans * nmaps
    # phase[pair][comp][hemisphere][m]
    phase = np.zeros((npairs, ncomp, 2, mmax + 1), np.complex128)
    cth = np.array([p[0].cth for p in geom.pairs])
    sth = np.array([p[0].sth for p in geom.pairs])
    ispair = np.array([p[1] is not None and p[1].nph > 0 for p in geom.pairs])
    mlim = np.array([get_mlim(lmax, spin, sth[i], cth[i]) for i in range(npairs)])

    # map2phase, sharp.c:672-715
    if analysis:
        for ip, (r1, r2) in enumerate(geom.pairs):
            for ic in range(ncomp):
                for h, r in enumerate((r1, r2)):
                    if r is None or r.nph <= 0:
                        continue
                    if flags & SHARP_NO_FFT:
                        wgt = (r.nph * r.weight) if (flags & SHARP_USE_WEIGHTS) else 1.0
                        if flags & SHARP_REAL_HARMONICS:
                            wgt *= SQRT_TWO
                        phase[ip, ic, h] = maps[ic][r.ofs + np.arange(mmax + 1) * r.stride] * wgt
                    else:
                        data = maps[ic][r.ofs + np.arange(r.nph) * r.stride].astype(np.float64)
                        phase[ip, ic, h] = ring2phase(r, data, mmax, flags)

    gen = Ylmgen(lmax, mmax, spin)
    for mi in range(nm):
        m = int(mval[mi])
        gen.prepare(m)
        act = mlim >= m
        if not act.any():
            continue
        c, s = cth[act], sth[act]
        # almtmp: alm2almtmp, sharp.c:481-545
        if not analysis:
            at = np.zeros((lmax + 1, ntrans * nalm), np.complex128)
            norm_m0 = SQRT_TWO if (flags & SHARP_REAL_HARMONICS) else 1.0
            for i in range(ntrans * nalm):
                vals = _alm_get(alm[i], ainfo, mi)
                fac = norm_l[m:] if (spin > 0 or deriv) else 1.0
                v = vals * fac
                if m == 0:
                    v = v.real * norm_m0
                at[m:, i] = v
        if spin == 0 and not deriv:
            lam = legendre_spin0(gen, m, c, s)  # (lmax+1, nact)
            par = ((np.arange(lmax + 1) - m) & 1) == 1
            even = lam.copy(); even[par] = 0
            odd = lam.copy(); odd[~par] = 0
            if not analysis:
                for i in range(ntrans):
                    p1 = at[:, i] @ even; p2 = at[:, i] @ odd
                    phase[act, i, 0, m] = p1 + p2
                    phase[act, i, 1, m] = np.where(ispair[act], p1 - p2, 0)
            else:
                for i in range(ntrans):
                    ph1 = phase[act, i, 0, m]
                    ph2 = np.where(ispair[act], phase[act, i, 1, m], 0)
                    res = even @ (ph1 + ph2) + odd @ (ph1 - ph2)
                    _alm_add(alm[i], ainfo, mi, res[m:], norm_l, spin, deriv, flags)
        else:
            rp, rm = legendre_spin(gen, m, c, s)
            lw = rp + rm; lx = rm - rp
            off = (np.arange(lmax + 1) - gen.mhi) & 1
            ev = (off == 0)[:, None]
            flip = ((gen.mhi - m + spin) & 1) == 1
            for j in range(ntrans):
                if not analysis:
                    if deriv:
                        a = at[:, j]
                        # saddstep_d, sharp_core_inc2.c:521-540
                        q_x = a @ np.where(ev, lw, 0), a @ np.where(~ev, lw, 0)   # into px (p1 for even)
                        u_y = (-1j * a) @ np.where(ev, lx, 0), (-1j * a) @ np.where(~ev, lx, 0)
                        q1, q2 = q_x[0], q_x[1]
                        u1, u2 = u_y[1], u_y[0]
                    else:
                        G = at[:, 2 * j]; C = at[:, 2 * j + 1]
                        # saddstep, sharp_core_inc2.c:282-306
                        qx = (G @ np.where(ev, lw, 0), G @ np.where(~ev, lw, 0))
                        ux = (C @ np.where(ev, lw, 0), C @ np.where(~ev, lw, 0))
                        # py.q += i*C*lx, py.u += -i*G*lx (vfmseq is a -= b*c)
                        qy = ((1j * C) @ np.where(ev, lx, 0), (1j * C) @ np.where(~ev, lx, 0))
                        uy = ((-1j * G) @ np.where(ev, lx, 0), (-1j * G) @ np.where(~ev, lx, 0))
                        # even offsets: px=p1, py=p2; odd offsets: px=p2, py=p1
                        q1 = qx[0] + qy[1]; q2 = qx[1] + qy[0]
                        u1 = ux[0] + uy[1]; u2 = ux[1] + uy[0]
                    phase[act, 2 * j, 0, m] = q1 + q2
                    phase[act, 2 * j + 1, 0, m] = u1 + u2
                    sq = np.where(ispair[act], q1 - q2, 0)
                    su = np.where(ispair[act], u1 - u2, 0)
                    if flip:
                        sq, su = -sq, -su
                    phase[act, 2 * j, 1, m] = sq
                    phase[act, 2 * j + 1, 1, m] = su
                else:
                    pq1 = phase[act, 2 * j, 0, m]; pu1 = phase[act, 2 * j + 1, 0, m]
                    pq2 = np.where(ispair[act], phase[act, 2 * j, 1, m], 0)
                    pu2 = np.where(ispair[act], phase[act, 2 * j + 1, 1, m], 0)
                    if flip:
                        pq2, pu2 = -pq2, -pu2
                    P1q, P1u = pq1 + pq2, pu1 + pu2
                    P2q, P2u = pq1 - pq2, pu1 - pu2
                    # saddstep2, sharp_core_inc2.c:338-364; px=p1 for even offsets
                    lwe = np.where(ev, lw, 0); lwo = np.where(~ev, lw, 0)
                    lxe = np.where(ev, lx, 0); lxo = np.where(~ev, lx, 0)
                    # agr -= py.ui*lx, agi += py.ur*lx  ->  G += i*lx*py.u
                    # acr += py.qi*lx, aci -= py.qr*lx  ->  C += -i*lx*py.q
                    G = lwe @ P1q + lwo @ P2q + 1j * (lxe @ P2u + lxo @ P1u)
                    C = lwe @ P1u + lwo @ P2u - 1j * (lxe @ P2q + lxo @ P1q)
                    _alm_add(alm[2 * j], ainfo, mi, G[m:], norm_l, spin, deriv, flags)
                    _alm_add(alm[2 * j + 1], ainfo, mi, C[m:], norm_l, spin, deriv, flags)

    # phase2map, sharp.c:717-760
    if not analysis:
        for ip, (r1, r2) in enumerate(geom.pairs):
            for ic in range(ncomp):
                for h, r in enumerate((r1, r2)):
                    if r is None or r.nph <= 0:
                        continue
                    if flags & SHARP_NO_FFT:
                        wgt = (r.nph * r.weight) if (flags & SHARP_USE_WEIGHTS) else 1.0
                        if flags & SHARP_REAL_HARMONICS:
                            wgt *= SQRT_ONE_HALF
                        maps[ic][r.ofs + np.arange(mmax + 1) * r.stride] += wgt * phase[ip, ic, h]
                    else:
                        vals = phase2ring(r, phase[ip, ic, h], mmax, flags)
                        maps[ic][r.ofs + np.arange(r.nph) * r.stride] += vals


def _alm_index(ainfo, mi, l, m):
    return ainfo.mvstart[mi] + ainfo.stride * l


def _alm_get(a, ainfo, mi):
    """a_lm for l=m..lmax at index mi (SHARP_PACKED: sharp_lowlevel.h:89)."""
    m = int(ainfo.mval[mi]); l = np.arange(m, ainfo.lmax + 1)
    if ainfo.flags & SHARP_PACKED:
        flat = a.view(np.float64)
        if m == 0:
            return flat[ainfo.mvstart[mi] + l * ainfo.stride].astype(np.complex128)
        idx = ainfo.mvstart[mi] + 2 * l * ainfo.stride
        return flat[idx] + 1j * flat[idx + 1]
    return a[ainfo.mvstart[mi] + l * ainfo.stride]


def _alm_clear(a, ainfo):
    for mi in range(ainfo.nm):
        m = int(ainfo.mval[mi]); l = np.arange(m, ainfo.lmax + 1)
        if ainfo.flags & SHARP_PACKED:
            flat = a.view(np.float64)
            if m == 0:
                flat[ainfo.mvstart[mi] + l * ainfo.stride] = 0
            else:
                idx = ainfo.mvstart[mi] + 2 * l * ainfo.stride
                flat[idx] = 0; flat[idx + 1] = 0
        else:
            a[ainfo.mvstart[mi] + l * ainfo.stride] = 0


def _alm_add(a, ainfo, mi, vals, norm_l, spin, deriv, flags):
    """almtmp2alm, libsharp/sharp.c:547-606."""
    m = int(ainfo.mval[mi]); l = np.arange(m, ainfo.lmax + 1)
    fac = norm_l[m:] if (spin > 0 or deriv) else 1.0
    v = vals * fac
    if m == 0:
        v = v.real * (SQRT_ONE_HALF if (flags & SHARP_REAL_HARMONICS) else 1.0)
    if ainfo.flags & SHARP_PACKED:
        flat = a.view(np.float64)
        if m == 0:
            flat[ainfo.mvstart[mi] + l * ainfo.stride] += np.real(v)
        else:
            idx = ainfo.mvstart[mi] + 2 * l * ainfo.stride
            flat[idx] += v.real; flat[idx + 1] += v.imag
    else:
        a[ainfo.mvstart[mi] + l * ainfo.stride] += v


# ---------------------------------------------------------------------------
# Convenience: the reference test suite's seeded a_lm (sharp_testsuite.c:53-82)
# ---------------------------------------------------------------------------
def testsuite_random_alm(lmax, mmax, spin, cnt):
    """random_alm with the in-file LCG drand, sharp_testsuite.c:53-82
    (triangular layout, stride 1)."""
    ainfo = triangular_alm_info(lmax, mmax)
    out = np.zeros(nalm_triangular(lmax, mmax), np.complex128)
    for m in range(mmax + 1):
        state = (1234567 * cnt + 8912 * m) & 0xFFFFFFFF
        state = state - (1 << 32) if state >= (1 << 31) else state
        for l in range(m, lmax + 1):
            idx = ainfo.mvstart[m] + l
            if l < spin and m < spin:
                out[idx] = 0
            else:
                state = _lcg(state); rv = -1 + 2 * state / (0x7fffffff + 1.0)
                iv = 0.0
                if m != 0:
                    state = _lcg(state); iv = -1 + 2 * state / (0x7fffffff + 1.0)
                out[idx] = rv + 1j * iv
    return out


def _lcg(state):
    # (state*1103515245 + 12345) & 0x7fffffff with C int wrap-around
    return ((state * 1103515245 + 12345) & 0xFFFFFFFF) & 0x7fffffff
