"""ctypes binding of the reference libsharp built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY (checker and CPU baseline; never the product path).
The library is zonca/planck-levelS's own c_utils + libfftpack + libsharp
compiled from its sources with every exported symbol renamed ``ref_*``.
Struct layouts follow libsharp/sharp_lowlevel.h:43-86.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libsharp_ref.so")


class RingInfo(C.Structure):
    _fields_ = [("theta", C.c_double), ("phi0", C.c_double), ("weight", C.c_double),
                ("cth", C.c_double), ("sth", C.c_double), ("ofs", C.c_ssize_t),
                ("nph", C.c_int), ("stride", C.c_int)]


class RingPair(C.Structure):
    _fields_ = [("r1", RingInfo), ("r2", RingInfo)]


class GeomInfo(C.Structure):
    _fields_ = [("pair", C.POINTER(RingPair)), ("npairs", C.c_int), ("nphmax", C.c_int)]


class AlmInfo(C.Structure):
    _fields_ = [("lmax", C.c_int), ("nm", C.c_int), ("mval", C.POINTER(C.c_int)),
                ("flags", C.c_int), ("mvstart", C.POINTER(C.c_ssize_t)),
                ("stride", C.c_ssize_t)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle`")
        _lib = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
        L = _lib
        L.ref_sharp_execute.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.POINTER(GeomInfo), C.POINTER(AlmInfo), C.c_int,
                                        C.c_int, C.POINTER(C.c_double),
                                        C.POINTER(C.c_ulonglong)]
        L.ref_sharp_execute.restype = None
        PG = C.POINTER(C.POINTER(GeomInfo))
        PA = C.POINTER(C.POINTER(AlmInfo))
        L.ref_sharp_make_weighted_healpix_geom_info.argtypes = [C.c_int, C.c_int, C.c_void_p, PG]
        for nm in ("gauss", "fejer1", "fejer2", "cc", "mw"):
            f = getattr(L, f"ref_sharp_make_{nm}_geom_info")
            f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, PG]
        L.ref_sharp_make_geom_info.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p, PG]
        L.ref_sharp_make_triangular_alm_info.argtypes = [C.c_int, C.c_int, C.c_int, PA]
        L.ref_sharp_make_rectangular_alm_info.argtypes = [C.c_int, C.c_int, C.c_int, PA]
        L.ref_sharp_make_general_alm_info.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p,
                                                      C.c_void_p, C.c_int, PA]
        L.ref_sharp_destroy_geom_info.argtypes = [C.POINTER(GeomInfo)]
        L.ref_sharp_destroy_alm_info.argtypes = [C.POINTER(AlmInfo)]
        L.ref_sharp_get_mlim.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
        L.ref_sharp_get_mlim.restype = C.c_int
    return _lib


class Geom:
    """Owns a reference sharp_geom_info."""

    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        if self.ptr and _lib is not None:
            _lib.ref_sharp_destroy_geom_info(self.ptr)
            self.ptr = None

    @property
    def npairs(self):
        return self.ptr.contents.npairs

    def npix(self):
        g = self.ptr.contents
        n = 0
        for i in range(g.npairs):
            n += g.pair[i].r1.nph + max(g.pair[i].r2.nph, 0)
        return n


class Alm:
    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        if self.ptr and _lib is not None:
            _lib.ref_sharp_destroy_alm_info(self.ptr)
            self.ptr = None


def healpix(nside, weight=None, stride=1) -> Geom:
    p = C.POINTER(GeomInfo)()
    w = None
    if weight is not None:
        w = np.ascontiguousarray(weight, np.float64)
    lib().ref_sharp_make_weighted_healpix_geom_info(
        nside, stride, None if w is None else w.ctypes.data, C.byref(p))
    g = Geom(p); g._keep = w
    return g


def grid(kind, nrings, nphi, phi0=0.0, stride_lon=1, stride_lat=None) -> Geom:
    p = C.POINTER(GeomInfo)()
    getattr(lib(), f"ref_sharp_make_{kind}_geom_info")(
        nrings, nphi, phi0, stride_lon, nphi if stride_lat is None else stride_lat, C.byref(p))
    return Geom(p)


def general(nph, ofs, stride, phi0, theta, wgt=None) -> Geom:
    nph = np.ascontiguousarray(nph, np.int32); ofs = np.ascontiguousarray(ofs, np.intp)
    stride = np.ascontiguousarray(stride, np.int32); phi0 = np.ascontiguousarray(phi0, np.float64)
    theta = np.ascontiguousarray(theta, np.float64)
    w = None if wgt is None else np.ascontiguousarray(wgt, np.float64)
    p = C.POINTER(GeomInfo)()
    lib().ref_sharp_make_geom_info(len(nph), nph.ctypes.data, ofs.ctypes.data, stride.ctypes.data,
                                   phi0.ctypes.data, theta.ctypes.data,
                                   None if w is None else w.ctypes.data, C.byref(p))
    return Geom(p)


def triangular(lmax, mmax, stride=1) -> Alm:
    p = C.POINTER(AlmInfo)()
    lib().ref_sharp_make_triangular_alm_info(lmax, mmax, stride, C.byref(p))
    return Alm(p)


def general_alm(lmax, mval, mvstart, stride=1, flags=0) -> Alm:
    mval = np.ascontiguousarray(mval, np.int32); mvstart = np.ascontiguousarray(mvstart, np.intp)
    p = C.POINTER(AlmInfo)()
    lib().ref_sharp_make_general_alm_info(lmax, len(mval), stride, mval.ctypes.data,
                                          mvstart.ctypes.data, flags, C.byref(p))
    return Alm(p)


def execute(jtype, spin, alms, maps, geom: Geom, ainfo: Alm, ntrans, flags):
    """Calls ref_sharp_execute on lists of numpy arrays; returns (time, opcnt)."""
    aptr = (C.c_void_p * len(alms))(*[a.ctypes.data for a in alms])
    mptr = (C.c_void_p * len(maps))(*[m.ctypes.data for m in maps])
    t = C.c_double(0.0); op = C.c_ulonglong(0)
    lib().ref_sharp_execute(jtype, spin, aptr, mptr, geom.ptr, ainfo.ptr, ntrans, flags,
                            C.byref(t), C.byref(op))
    return t.value, op.value


def get_mlim(lmax, spin, sth, cth):
    return lib().ref_sharp_get_mlim(lmax, spin, sth, cth)
