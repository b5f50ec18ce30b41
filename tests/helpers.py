"""Shared test utilities: seeded inputs with the benchmark distributions and
error metrics.  Inputs are generated once and handed to both the GPU engine
and the oracle."""
from __future__ import annotations

import numpy as np

ARCMIN = np.pi / 10800.0


def cl_spectrum(lmax, beam_arcmin=0.0):
    """C_l = 1/(l+1)^2 * exp(-l(l+1) sigma^2), l<2 zeroed (sigma = beam taken
    literally as the Gaussian sigma, in arcmin)."""
    l = np.arange(lmax + 1, dtype=np.float64)
    cl = 1.0 / (l + 1.0) ** 2
    if beam_arcmin:
        s = beam_arcmin * ARCMIN
        cl *= np.exp(-l * (l + 1) * s * s)
    cl[:2] = 0.0
    return cl


def random_alm(lmax, mmax=None, seed=0, cl=None, rng=None):
    """Triangular m-major a_lm: sqrt(C_l/2)(N+iN) for m>0, sqrt(C_l) N (real)
    for m=0."""
    mmax = lmax if mmax is None else mmax
    rng = np.random.default_rng(seed) if rng is None else rng
    if cl is None:
        cl = cl_spectrum(lmax)
    out = []
    for m in range(mmax + 1):
        l = np.arange(m, lmax + 1)
        if m == 0:
            v = np.sqrt(cl[l]) * rng.standard_normal(len(l)) + 0j
        else:
            v = np.sqrt(cl[l] / 2) * (rng.standard_normal(len(l)) + 1j * rng.standard_normal(len(l)))
        out.append(v)
    return np.concatenate(out).astype(np.complex128)


def uniform_alm(lmax, mmax=None, seed=0, spin=0):
    """Uniform(-1,1) a_lm (m=0 real), zero where l<spin."""
    mmax = lmax if mmax is None else mmax
    rng = np.random.default_rng(seed)
    out = []
    for m in range(mmax + 1):
        l = np.arange(m, lmax + 1)
        re = rng.uniform(-1, 1, len(l))
        im = np.zeros(len(l)) if m == 0 else rng.uniform(-1, 1, len(l))
        v = re + 1j * im
        v[l < spin] = 0
        out.append(v)
    return np.concatenate(out)


def rel_l2(a, b):
    a = np.asarray(a); b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


def npix_healpix(nside):
    return 12 * nside * nside
