"""Python mirror of the libsharp C interface, backed by libsharp_b200.so.

The shared library next to this file implements libsharp's ``sharp_execute``
ABI (zonca/planck-levelS libsharp/sharp_lowlevel.h) on the GPU.  This module
binds it with ctypes using the same names and argument meaning as the C API,
so host code reads like the reference's own callers (sharp_cxx.h,
sharp_testsuite.c).  There is no CPU fallback: importing fails loudly when the
library is missing, and the library fails loudly without a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsharp_b200.so")

# job types and flags (sharp_lowlevel.h / sharp_b200.h)
SHARP_YtW = SHARP_MAP2ALM = 0
SHARP_Y = SHARP_ALM2MAP = 1
SHARP_Yt = 2
SHARP_WY = 3
SHARP_ALM2MAP_DERIV1 = 4
SHARP_DP = 1 << 4
SHARP_ADD = 1 << 5
SHARP_REAL_HARMONICS = 1 << 6
SHARP_NO_FFT = 1 << 7
SHARP_ADJOINT = 1 << 8
SHARP_MIXED = 1 << 9
SHARP_SUBTRACT = 1 << 10
SHARP_PACKED = 1


class sharp_ringinfo(C.Structure):
    _fields_ = [("theta", C.c_double), ("phi0", C.c_double), ("weight", C.c_double),
                ("cth", C.c_double), ("sth", C.c_double), ("ofs", C.c_ssize_t),
                ("nph", C.c_int), ("stride", C.c_int)]


class sharp_ringpair(C.Structure):
    _fields_ = [("r1", sharp_ringinfo), ("r2", sharp_ringinfo)]


class sharp_geom_info(C.Structure):
    _fields_ = [("pair", C.POINTER(sharp_ringpair)), ("npairs", C.c_int), ("nphmax", C.c_int)]


class sharp_alm_info(C.Structure):
    _fields_ = [("lmax", C.c_int), ("nm", C.c_int), ("mval", C.POINTER(C.c_int)),
                ("flags", C.c_int), ("mvstart", C.POINTER(C.c_ssize_t)),
                ("stride", C.c_ssize_t)]


if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python planck-levels_b200/build.py` "
        "(the GPU engine has no CPU fallback)")

_lib = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
_PG = C.POINTER(C.POINTER(sharp_geom_info))
_PA = C.POINTER(C.POINTER(sharp_alm_info))
_lib.sharp_execute.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                               C.POINTER(sharp_geom_info), C.POINTER(sharp_alm_info), C.c_int,
                               C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_ulonglong)]
_lib.sharp_execute.restype = None
_lib.sharp_b200_execute_device.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                           C.POINTER(sharp_geom_info),
                                           C.POINTER(sharp_alm_info), C.c_int, C.c_int,
                                           C.c_void_p, C.POINTER(C.c_double),
                                           C.POINTER(C.c_ulonglong)]
_lib.sharp_b200_execute_device.restype = None
_lib.sharp_make_weighted_healpix_geom_info.argtypes = [C.c_int, C.c_int, C.c_void_p, _PG]
for _nm in ("gauss", "fejer1", "fejer2", "cc", "mw"):
    getattr(_lib, f"sharp_make_{_nm}_geom_info").argtypes = [C.c_int, C.c_int, C.c_double,
                                                             C.c_int, C.c_int, _PG]
_lib.sharp_make_geom_info.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, _PG]
_lib.sharp_destroy_geom_info.argtypes = [C.POINTER(sharp_geom_info)]
_lib.sharp_b200_make_subset_geom_info.argtypes = [C.POINTER(sharp_geom_info), C.c_void_p, C.c_int,
                                                  _PG]
_lib.sharp_b200_make_subset_geom_info.restype = C.c_int
_lib.sharp_get_mlim.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
_lib.sharp_get_mlim.restype = C.c_int
_lib.sharp_make_triangular_alm_info.argtypes = [C.c_int, C.c_int, C.c_int, _PA]
_lib.sharp_make_rectangular_alm_info.argtypes = [C.c_int, C.c_int, C.c_int, _PA]
_lib.sharp_make_alm_info.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, _PA]
_lib.sharp_make_general_alm_info.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                             C.c_int, _PA]
_lib.sharp_destroy_alm_info.argtypes = [C.POINTER(sharp_alm_info)]
_lib.sharp_alm_index.argtypes = [C.POINTER(sharp_alm_info), C.c_int, C.c_int]
_lib.sharp_alm_index.restype = C.c_ssize_t
_lib.sharp_b200_last_error.restype = C.c_char_p
_lib.sharp_b200_set_abort_on_error.argtypes = [C.c_int]
_lib.sharp_set_chunksize_min.argtypes = [C.c_int]
_lib.sharp_set_nchunks_max.argtypes = [C.c_int]


def lib():
    """The loaded ctypes library (for callers that bind extra symbols)."""
    return _lib


_lib.sharp_b200_workspace_bytes.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
_lib.sharp_b200_workspace_bytes.restype = C.c_int


def workspace_bytes():
    """(reserved, used) bytes of the library's workspace pool on the current
    device: freed workspace stays reserved for the next job until
    sharp_b200_release_cache().  (0, 0) before the first job."""
    r, u = C.c_ulonglong(0), C.c_ulonglong(0)
    _lib.sharp_b200_workspace_bytes(C.byref(r), C.byref(u))
    return r.value, u.value


_lib.sharp_b200_check_device_errors.argtypes = [C.c_void_p]
_lib.sharp_b200_check_device_errors.restype = C.c_int


def check_device_errors(stream=None) -> None:
    """sharp_b200_check_device_errors: waits for ``stream`` (a
    torch.cuda.Stream; default torch's current stream) and raises SharpError
    if a SHARP_MIXED transform enqueued there gave up on a bounded wait or the
    stream failed."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    _lib.sharp_b200_check_device_errors(C.c_void_p(stream.cuda_stream))
    _check()


def last_error() -> str:
    return _lib.sharp_b200_last_error().decode()


def clear_error() -> None:
    _lib.sharp_b200_clear_error()


def set_abort_on_error(on: bool) -> None:
    _lib.sharp_b200_set_abort_on_error(1 if on else 0)


class SharpError(RuntimeError):
    pass


def _check():
    msg = last_error()
    if msg:
        clear_error()
        raise SharpError(msg)


# ---------------------------------------------------------------------------
# Geometry and a_lm layout objects (sharp_geomhelpers.h, sharp_almhelpers.h)
# ---------------------------------------------------------------------------
class Geometry:
    """Owns a ``sharp_geom_info``; ``pairs`` exposes the pair array."""

    def __init__(self, ptr):
        self.ptr = ptr

    # the destructor is bound at class creation: module globals may already be
    # cleared when objects are collected at interpreter exit
    def __del__(self, _destroy=_lib.sharp_destroy_geom_info):
        p = getattr(self, "ptr", None)
        if p:
            _destroy(p)
            self.ptr = None

    @property
    def npairs(self) -> int:
        return self.ptr.contents.npairs

    @property
    def nphmax(self) -> int:
        return self.ptr.contents.nphmax

    def pair(self, i) -> sharp_ringpair:
        return self.ptr.contents.pair[i]

    def npix(self) -> int:
        g = self.ptr.contents
        return sum(g.pair[i].r1.nph + max(g.pair[i].r2.nph, 0) for i in range(g.npairs))

    def subset(self, pairs) -> "Geometry":
        """sharp_b200_make_subset_geom_info: a geometry of the ring pairs
        ``pairs`` (indices into this geometry's pair array)."""
        idx = np.ascontiguousarray(pairs, np.int32)
        p = C.POINTER(sharp_geom_info)()
        rc = _lib.sharp_b200_make_subset_geom_info(self.ptr, idx.ctypes.data, len(idx), C.byref(p))
        if rc != 0:
            _check()
        return Geometry(p)

    @classmethod
    def healpix(cls, nside: int, weight=None, stride: int = 1) -> "Geometry":
        p = C.POINTER(sharp_geom_info)()
        w = None if weight is None else np.ascontiguousarray(weight, np.float64)
        _lib.sharp_make_weighted_healpix_geom_info(nside, stride,
                                                   None if w is None else w.ctypes.data,
                                                   C.byref(p))
        return cls(p)

    @classmethod
    def grid(cls, kind: str, nrings: int, nphi: int, phi0: float = 0.0,
             stride_lon: int = 1, stride_lat: int | None = None) -> "Geometry":
        """kind in gauss, fejer1 (= ecp), fejer2, cc, mw."""
        kind = "fejer1" if kind == "ecp" else kind
        p = C.POINTER(sharp_geom_info)()
        getattr(_lib, f"sharp_make_{kind}_geom_info")(
            nrings, nphi, phi0, stride_lon, nphi if stride_lat is None else stride_lat,
            C.byref(p))
        return cls(p)

    @classmethod
    def general(cls, nph, ofs, stride, phi0, theta, wgt=None) -> "Geometry":
        nph = np.ascontiguousarray(nph, np.int32)
        ofs = np.ascontiguousarray(ofs, np.intp)
        stride = np.ascontiguousarray(stride, np.int32)
        phi0 = np.ascontiguousarray(phi0, np.float64)
        theta = np.ascontiguousarray(theta, np.float64)
        w = None if wgt is None else np.ascontiguousarray(wgt, np.float64)
        p = C.POINTER(sharp_geom_info)()
        _lib.sharp_make_geom_info(len(nph), nph.ctypes.data, ofs.ctypes.data, stride.ctypes.data,
                                  phi0.ctypes.data, theta.ctypes.data,
                                  None if w is None else w.ctypes.data, C.byref(p))
        return cls(p)


class AlmInfo:
    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self, _destroy=_lib.sharp_destroy_alm_info):
        p = getattr(self, "ptr", None)
        if p:
            _destroy(p)
            self.ptr = None

    @property
    def lmax(self):
        return self.ptr.contents.lmax

    @property
    def nm(self):
        return self.ptr.contents.nm

    def index(self, l, mi):
        return _lib.sharp_alm_index(self.ptr, l, mi)

    def nalm(self) -> int:
        a = self.ptr.contents
        return sum(a.lmax - a.mval[i] + 1 for i in range(a.nm))

    @classmethod
    def triangular(cls, lmax: int, mmax: int | None = None, stride: int = 1) -> "AlmInfo":
        p = C.POINTER(sharp_alm_info)()
        _lib.sharp_make_triangular_alm_info(lmax, lmax if mmax is None else mmax, stride,
                                            C.byref(p))
        return cls(p)

    @classmethod
    def rectangular(cls, lmax: int, mmax: int | None = None, stride: int = 1) -> "AlmInfo":
        p = C.POINTER(sharp_alm_info)()
        _lib.sharp_make_rectangular_alm_info(lmax, lmax if mmax is None else mmax, stride,
                                             C.byref(p))
        return cls(p)

    @classmethod
    def general(cls, lmax, mval, mvstart, stride=1, flags=0) -> "AlmInfo":
        mval = np.ascontiguousarray(mval, np.int32)
        mvstart = np.ascontiguousarray(mvstart, np.intp)
        p = C.POINTER(sharp_alm_info)()
        _lib.sharp_make_general_alm_info(lmax, len(mval), stride, mval.ctypes.data,
                                         mvstart.ctypes.data, flags, C.byref(p))
        return cls(p)


def nalm_triangular(lmax: int, mmax: int | None = None) -> int:
    mmax = lmax if mmax is None else mmax
    return ((mmax + 1) * (mmax + 2)) // 2 + (mmax + 1) * (lmax - mmax)


def set_chunksize_min(v: int) -> None:
    _lib.sharp_set_chunksize_min(v)


def set_nchunks_max(v: int) -> None:
    _lib.sharp_set_nchunks_max(v)


# ---------------------------------------------------------------------------
# sharp_execute on host arrays, sharp_b200_execute_device on torch tensors
# ---------------------------------------------------------------------------
def execute(jtype: int, spin: int, alm, maps, geom: Geometry, ainfo: AlmInfo,
            ntrans: int = 1, flags: int = SHARP_DP):
    """sharp_execute on lists of C-contiguous numpy arrays (written in place).

    Returns (wall time in s, operation count)."""
    aptr = (C.c_void_p * len(alm))(*[a.ctypes.data for a in alm])
    mptr = (C.c_void_p * len(maps))(*[m.ctypes.data for m in maps])
    t = C.c_double(0.0)
    op = C.c_ulonglong(0)
    _lib.sharp_execute(jtype, spin, aptr, mptr, geom.ptr, ainfo.ptr, ntrans, flags,
                       C.byref(t), C.byref(op))
    _check()
    return t.value, op.value


def execute_device(jtype: int, spin: int, alm, maps, geom: Geometry, ainfo: AlmInfo,
                   ntrans: int = 1, flags: int = SHARP_DP, stream=None):
    """sharp_b200_execute_device on lists of CUDA tensors (contiguous).

    ``stream`` is a torch.cuda.Stream (default: torch's current stream); the
    work is enqueued there without host synchronisation."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    aptr = (C.c_void_p * len(alm))(*[a.data_ptr() for a in alm])
    mptr = (C.c_void_p * len(maps))(*[m.data_ptr() for m in maps])
    op = C.c_ulonglong(0)
    _lib.sharp_b200_execute_device(jtype, spin, aptr, mptr, geom.ptr, ainfo.ptr, ntrans, flags,
                                   C.c_void_p(stream.cuda_stream), None, C.byref(op))
    _check()
    return op.value


class sharp_b200_job(C.Structure):
    _fields_ = [("type", C.c_int), ("spin", C.c_int), ("alm", C.c_void_p), ("map", C.c_void_p),
                ("geom_info", C.POINTER(sharp_geom_info)),
                ("alm_info", C.POINTER(sharp_alm_info)), ("ntrans", C.c_int), ("flags", C.c_int)]


_lib.sharp_b200_execute_batch.argtypes = [C.POINTER(sharp_b200_job), C.c_int, C.c_int,
                                          C.c_void_p, C.POINTER(C.c_ulonglong)]
_lib.sharp_b200_execute_batch.restype = C.c_int


def _job_array(jobs, device):
    """sharp_b200_job array of the job tuples (and the pointer arrays it uses)."""
    keep = []
    arr = (sharp_b200_job * max(len(jobs), 1))()
    for i, (jt, spin, alm, maps, geom, ainfo, nt, fl) in enumerate(jobs):
        ptr = (lambda a: a.data_ptr()) if device else (lambda a: a.ctypes.data)
        aptr = (C.c_void_p * len(alm))(*[ptr(a) for a in alm])
        mptr = (C.c_void_p * len(maps))(*[ptr(m) for m in maps])
        keep += [aptr, mptr]
        arr[i] = sharp_b200_job(jt, spin, C.cast(aptr, C.c_void_p), C.cast(mptr, C.c_void_p),
                                geom.ptr, ainfo.ptr, nt, fl)
    return arr, keep


_lib.sharp_b200_batch_groups.argtypes = [C.POINTER(sharp_b200_job), C.c_int, C.c_int,
                                         C.POINTER(C.c_int)]
_lib.sharp_b200_batch_groups.restype = C.c_int


def batch_groups(jobs, device: bool = False):
    """sharp_b200_batch_groups: how ``execute_batch`` would merge ``jobs``
    (same tuples); returns the group index of every job.  Host work only."""
    arr, keep = _job_array(jobs, device)
    of = (C.c_int * max(len(jobs), 1))()
    n = _lib.sharp_b200_batch_groups(arr, len(jobs), 1 if device else 0, of)
    _check()
    assert n >= 0
    return [of[i] for i in range(len(jobs))]


def execute_batch(jobs, device: bool = False, stream=None):
    """sharp_b200_execute_batch: ``jobs`` is a list of tuples
    (jtype, spin, alm, maps, geom, ainfo, ntrans, flags) with alm/maps lists
    of numpy arrays (device=False) or CUDA tensors (device=True), as in
    ``execute`` / ``execute_device``.  Compatible jobs are merged into one
    batched job.  With host arrays the jobs take effect in list order (a
    job may read arrays an earlier job writes, e.g. the alm2map and map2alm
    halves of a round trip; only consecutive jobs merge); with device arrays
    the jobs must be independent.  Returns (number of merged jobs, operation
    count)."""
    arr, keep = _job_array(jobs, device)
    st = None
    if device:
        import torch
        st = C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
    op = C.c_ulonglong(0)
    n = _lib.sharp_b200_execute_batch(arr, len(jobs), 1 if device else 0, st, C.byref(op))
    _check()
    return n, op.value
