"""The allocation-free spin-0 synthesis, called through the C ABI.

sharp_b200_alm2map_noalloc exists for callers that cannot call cudaMalloc
when they need a transform (their GPU memory belongs to another allocator,
or they forbid allocation after start-up); it keeps all scratch in one fixed
32 MiB device array.  Its maps must equal those of the regular device entry
point, call after call, and problems that do not fit the array must be
refused with an explanation instead of failing later.  This file is collected
last so that a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

import sharp_b200 as sb
from helpers import random_alm, rel_l2

pytestmark = pytest.mark.gpu


def _entry():
    f = sb.lib().sharp_b200_alm2map_noalloc
    f.argtypes = [C.POINTER(sb.sharp_geom_info), C.POINTER(sb.sharp_alm_info), C.c_void_p,
                  C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("geo", [("healpix", 64, 128), ("healpix", 128, 256),
                                 ("gauss", 65, 131, 64)])
def test_noalloc_matches_device_entry_twice(geo):
    import torch
    f = _entry()
    if geo[0] == "healpix":
        g, lmax = sb.Geometry.healpix(geo[1]), geo[2]
    else:
        g, lmax = sb.Geometry.grid("gauss", geo[1], geo[2]), geo[3]
    a = sb.AlmInfo.triangular(lmax)
    npix = g.npix()
    stream = torch.cuda.current_stream()
    for seed in (1, 2):  # two calls in a row, different inputs
        alm = torch.from_numpy(random_alm(lmax, seed=seed).view(np.float64).copy()).cuda()
        want = torch.zeros(npix, dtype=torch.float64, device="cuda")
        sb.execute_device(sb.SHARP_ALM2MAP, 0, [alm], [want], g, a, 1, sb.SHARP_DP)
        got = torch.full((npix,), 7.0, dtype=torch.float64, device="cuda")
        rc = f(g.ptr, a.ptr, C.c_void_p(alm.data_ptr()), C.c_void_p(got.data_ptr()),
               C.c_void_p(stream.cuda_stream))
        assert rc == 0, sb.last_error()
        torch.cuda.synchronize()
        assert rel_l2(got.cpu().numpy(), want.cpu().numpy()) < 1e-12


def test_noalloc_refuses_problems_above_its_scratch():
    import torch
    f = _entry()
    g, a = sb.Geometry.healpix(1024), sb.AlmInfo.triangular(2048)
    alm = torch.zeros(2 * sb.nalm_triangular(2048), dtype=torch.float64, device="cuda")
    mp = torch.zeros(12 * 1024 ** 2, dtype=torch.float64, device="cuda")
    sb.clear_error()
    rc = f(g.ptr, a.ptr, C.c_void_p(alm.data_ptr()), C.c_void_p(mp.data_ptr()),
           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -1
    assert "MiB of scratch" in sb.last_error()
    sb.clear_error()


def test_noalloc_allocates_no_device_memory():
    # the point of the entry point: after a first call on the device (which
    # looks up the array's address and loads the kernels), further calls
    # leave the library's workspace pool and the device's free memory exactly
    # as they were
    import torch
    f = _entry()
    nside, lmax = 128, 256
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    alm = torch.from_numpy(random_alm(lmax, seed=3).view(np.float64).copy()).cuda()
    got = torch.zeros(12 * nside * nside, dtype=torch.float64, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (g.ptr, a.ptr, C.c_void_p(alm.data_ptr()), C.c_void_p(got.data_ptr()), st)
    assert f(*args) == 0, sb.last_error()
    torch.cuda.synchronize()
    pool0 = sb.workspace_bytes()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        assert f(*args) == 0, sb.last_error()
    torch.cuda.synchronize()
    assert sb.workspace_bytes() == pool0
    assert torch.cuda.mem_get_info()[0] == free0
