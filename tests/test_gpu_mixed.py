"""Mixed-precision batched transforms (SHARP_MIXED): FP64 recurrence, exact
int8 tcgen05 Legendre contraction, against the FP64 engine and the
reference.

Tolerance: 1e-6 relative L2 against the FP64 result, the bar stated for the
mixed-precision form (FP64 recurrence seeds, tensor-core contraction)."""
import numpy as np
import pytest

import sharp_b200 as sb
from helpers import random_alm, rel_l2, uniform_alm

pytestmark = pytest.mark.gpu
DP = sb.SHARP_DP
MIXED = sb.SHARP_MIXED
TOL = 1e-6


def _geom(spec):
    if spec[0] == "healpix":
        return sb.Geometry.healpix(spec[1])
    return sb.Geometry.grid(*spec)


def _synth_both(spec, lmax, mmax, ntrans, alm_fn, flags=0, init=None, spin=0):
    """alm2map of the same inputs through the FP64 and the mixed path; for
    spin > 0 alm_fn(i) gives the i-th a_lm component (E, B interleaved per
    transform) and each transform yields (Q, U)."""
    g = _geom(spec)
    a = sb.AlmInfo.triangular(lmax, mmax)
    npix = g.npix()
    ncomp = 1 if spin == 0 else 2
    alms = [alm_fn(i) for i in range(ntrans * ncomp)]
    m64 = [np.zeros(npix) if init is None else init[i].copy() for i in range(ntrans * ncomp)]
    mmx = [x.copy() for x in m64]
    sb.execute(sb.SHARP_ALM2MAP, spin, [x.copy() for x in alms], m64, g, a, ntrans, DP | flags)
    sb.execute(sb.SHARP_ALM2MAP, spin, [x.copy() for x in alms], mmx, g, a, ntrans,
               DP | MIXED | flags)
    return m64, mmx


@pytest.mark.parametrize("ntrans", [1, 2, 3, 5, 8, 16, 17])
def test_mixed_healpix_batches(ntrans):
    lmax = 96
    m64, mmx = _synth_both(("healpix", 48), lmax, lmax, ntrans,
                           lambda i: uniform_alm(lmax, seed=10 + i))
    for x, y in zip(mmx, m64):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spec,lmax,mmax", [
    (("gauss", 130, 259), 129, 129),
    (("gauss", 64, 128), 63, 40),       # mmax < lmax
    (("cc", 90, 171), 80, 80),          # poles on the grid
    (("healpix", 128), 300, 300),       # lmax > 2 nside
])
def test_mixed_geometries(spec, lmax, mmax):
    m64, mmx = _synth_both(spec, lmax, mmax, 4,
                           lambda i: random_alm(lmax, mmax, seed=3 + i))
    for x, y in zip(mmx, m64):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spin,ntrans", [(1, 1), (2, 1), (2, 2), (2, 3), (2, 4), (2, 7), (3, 2)])
def test_mixed_spin_batches(spin, ntrans):
    lmax = 96
    m64, mmx = _synth_both(("healpix", 48), lmax, lmax, ntrans,
                           lambda i: uniform_alm(lmax, seed=30 + i, spin=spin), spin=spin)
    for x, y in zip(mmx, m64):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spec,lmax,mmax", [
    (("gauss", 130, 259), 129, 129),
    (("gauss", 64, 128), 63, 40),
    (("cc", 90, 171), 80, 80),
])
def test_mixed_spin2_geometries(spec, lmax, mmax):
    m64, mmx = _synth_both(spec, lmax, mmax, 2,
                           lambda i: uniform_alm(lmax, mmax, seed=50 + i, spin=2), spin=2)
    for x, y in zip(mmx, m64):
        assert rel_l2(x, y) < TOL


def test_mixed_add_flag():
    lmax, nside = 64, 32
    rng = np.random.default_rng(7)
    init = [rng.standard_normal(12 * nside * nside) for _ in range(4)]
    m64, mmx = _synth_both(("healpix", nside), lmax, lmax, 4,
                           lambda i: uniform_alm(lmax, seed=20 + i), flags=sb.SHARP_ADD,
                           init=init)
    for x, y, z in zip(mmx, m64, init):
        assert rel_l2(x - z, y - z) < TOL


def test_mixed_against_reference():
    import ref
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    nside, lmax = 64, 128
    g, a = ref.healpix(nside), ref.triangular(lmax, lmax)
    alms = [random_alm(lmax, seed=40 + i) for i in range(8)]
    out_ref = [np.zeros(12 * nside * nside) for _ in alms]
    ref.execute(sb.SHARP_ALM2MAP, 0, [x.copy() for x in alms], out_ref, g, a, 8, DP)
    _, mmx = _synth_both(("healpix", nside), lmax, lmax, 8, lambda i: alms[i])
    for x, y in zip(mmx, out_ref):
        assert rel_l2(x, y) < TOL


def test_mixed_device_entry_high_lmax():
    # device-resident call at a size where the scaled (exponent-tracked)
    # regime of the recurrence matters: lmax 1500, small sin(theta) rings
    import torch
    nside, lmax, nt = 512, 1500, 16
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax, lmax)
    dev = torch.device("cuda:0")
    alms = [torch.from_numpy(random_alm(lmax, seed=60 + i)).to(dev) for i in range(nt)]
    ra = [torch.view_as_real(x).reshape(-1) for x in alms]
    m64 = [torch.zeros(12 * nside * nside, dtype=torch.float64, device=dev) for _ in range(nt)]
    mmx = [torch.zeros_like(x) for x in m64]
    sb.execute_device(sb.SHARP_ALM2MAP, 0, ra, m64, g, a, nt, DP)
    sb.execute_device(sb.SHARP_ALM2MAP, 0, ra, mmx, g, a, nt, DP | MIXED)
    torch.cuda.synchronize()
    for x, y in zip(mmx, m64):
        assert rel_l2(x.cpu().numpy(), y.cpu().numpy()) < TOL


# ---------------------------------------------------------------------------
# map2alm with SHARP_MIXED (tensor-core analysis, spin 0)
# ---------------------------------------------------------------------------
def _anal_both(spec, lmax, mmax, ntrans, seed=0, flags=0, init=None):
    g = _geom(spec)
    a = sb.AlmInfo.triangular(lmax, mmax)
    npix, nalm = g.npix(), sb.nalm_triangular(lmax, mmax)
    rng = np.random.default_rng(seed)
    maps = [rng.standard_normal(npix) for _ in range(ntrans)]
    o64 = [np.zeros(nalm, np.complex128) if init is None else init[i].copy()
           for i in range(ntrans)]
    omx = [x.copy() for x in o64]
    sb.execute(sb.SHARP_MAP2ALM, 0, o64, [x.copy() for x in maps], g, a, ntrans, DP | flags)
    sb.execute(sb.SHARP_MAP2ALM, 0, omx, [x.copy() for x in maps], g, a, ntrans,
               DP | MIXED | flags)
    return o64, omx


@pytest.mark.parametrize("ntrans", [1, 2, 3, 4, 5, 9])
def test_mixed_analysis_healpix_batches(ntrans):
    o64, omx = _anal_both(("healpix", 48), 96, 96, ntrans, seed=ntrans)
    for x, y in zip(omx, o64):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spec,lmax,mmax", [
    (("gauss", 130, 259), 129, 129),
    (("gauss", 64, 128), 63, 40),       # mmax < lmax
    (("cc", 90, 171), 80, 80),          # poles on the grid
    (("healpix", 128), 300, 300),       # lmax > 2 nside, several ring groups
    (("healpix", 160), 200, 200),       # more than 256 ring pairs per m
])
def test_mixed_analysis_geometries(spec, lmax, mmax):
    o64, omx = _anal_both(spec, lmax, mmax, 4, seed=11)
    for x, y in zip(omx, o64):
        assert rel_l2(x, y) < TOL


def test_mixed_analysis_add_flag():
    lmax = 64
    rng = np.random.default_rng(5)
    nalm = sb.nalm_triangular(lmax)
    init = [rng.standard_normal(nalm) + 1j * rng.standard_normal(nalm) for _ in range(3)]
    o64, omx = _anal_both(("healpix", 32), lmax, lmax, 3, seed=6, flags=sb.SHARP_ADD,
                          init=init)
    for x, y, z in zip(omx, o64, init):
        assert rel_l2(x - z, y - z) < TOL


def test_mixed_round_trip_against_reference():
    import ref
    if not ref.available():
        pytest.skip("reference library not built (make -C oracle)")
    nside, lmax = 64, 128
    g, a = ref.healpix(nside), ref.triangular(lmax, lmax)
    rng = np.random.default_rng(9)
    maps = [rng.standard_normal(12 * nside * nside) for _ in range(4)]
    out_ref = [np.zeros(sb.nalm_triangular(lmax), np.complex128) for _ in maps]
    ref.execute(sb.SHARP_MAP2ALM, 0, out_ref, [x.copy() for x in maps], g, a, 4, DP)
    gg, aa = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax, lmax)
    out = [np.zeros_like(x) for x in out_ref]
    sb.execute(sb.SHARP_MAP2ALM, 0, out, [x.copy() for x in maps], gg, aa, 4, DP | MIXED)
    for x, y in zip(out, out_ref):
        assert rel_l2(x, y) < TOL


def _anal_spin_both(spec, lmax, mmax, ntrans, spin, seed=0):
    g = _geom(spec)
    a = sb.AlmInfo.triangular(lmax, mmax)
    npix, nalm = g.npix(), sb.nalm_triangular(lmax, mmax)
    rng = np.random.default_rng(seed)
    maps = [rng.standard_normal(npix) for _ in range(2 * ntrans)]
    o64 = [np.zeros(nalm, np.complex128) for _ in range(2 * ntrans)]
    omx = [x.copy() for x in o64]
    sb.execute(sb.SHARP_MAP2ALM, spin, o64, [x.copy() for x in maps], g, a, ntrans, DP)
    sb.execute(sb.SHARP_MAP2ALM, spin, omx, [x.copy() for x in maps], g, a, ntrans, DP | MIXED)
    return o64, omx


@pytest.mark.parametrize("spin,ntrans", [(1, 1), (2, 1), (2, 2), (2, 3), (3, 2)])
def test_mixed_spin_analysis_batches(spin, ntrans):
    o64, omx = _anal_spin_both(("healpix", 48), 96, 96, ntrans, spin, seed=spin + ntrans)
    for x, y in zip(omx, o64):
        assert rel_l2(x, y) < TOL


@pytest.mark.parametrize("spec,lmax,mmax", [
    (("gauss", 130, 259), 129, 129),
    (("gauss", 64, 128), 63, 40),
    (("cc", 90, 171), 80, 80),
    (("healpix", 128), 300, 300),       # several 128-pair groups per m
])
def test_mixed_spin2_analysis_geometries(spec, lmax, mmax):
    o64, omx = _anal_spin_both(spec, lmax, mmax, 2, 2, seed=21)
    for x, y in zip(omx, o64):
        assert rel_l2(x, y) < TOL


def test_mixed_nside4096_lmax8192_round_trip():
    # the large polarised configuration: Nside 4096 (rings up to 16384 pixels),
    # lmax = mmax = 8192, spin 0 + 2, device-resident; mixed against FP64 in
    # both directions
    import torch
    nside, lmax = 4096, 8192
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax, lmax)
    dev = torch.device("cuda:0")
    npix = 12 * nside * nside
    for spin in (0, 2):
        nc = 1 if spin == 0 else 2
        alms = [torch.view_as_real(torch.from_numpy(
            random_alm(lmax, lmax, seed=80 + i)).to(dev)).reshape(-1) for i in range(nc)]
        m64 = [torch.zeros(npix, dtype=torch.float64, device=dev) for _ in range(nc)]
        mmx = [torch.zeros_like(x) for x in m64]
        sb.execute_device(sb.SHARP_ALM2MAP, spin, alms, m64, g, a, 1, DP)
        sb.execute_device(sb.SHARP_ALM2MAP, spin, alms, mmx, g, a, 1, DP | MIXED)
        a64 = [torch.zeros_like(x) for x in alms]
        amx = [torch.zeros_like(x) for x in alms]
        sb.execute_device(sb.SHARP_MAP2ALM, spin, a64, m64, g, a, 1, DP)
        sb.execute_device(sb.SHARP_MAP2ALM, spin, amx, m64, g, a, 1, DP | MIXED)
        torch.cuda.synchronize()
        for x, y in zip(mmx, m64):
            assert (torch.linalg.norm(x - y) / torch.linalg.norm(y)).item() < TOL
        for x, y in zip(amx, a64):
            assert (torch.linalg.norm(x - y) / torch.linalg.norm(y)).item() < TOL
        del alms, m64, mmx, a64, amx


@pytest.mark.parametrize("jtype,spin,flags", [
    (sb.SHARP_ALM2MAP, 2, DP | MIXED), (sb.SHARP_MAP2ALM, 2, DP | MIXED),
    (sb.SHARP_ALM2MAP, 0, DP), (sb.SHARP_MAP2ALM, 0, DP | MIXED)])
def test_host_arrays_in_pieces_equal_device_call(jtype, spin, flags):
    # a host-array job of several transforms runs in pieces with overlapped
    # copies (pinned buffers here); its outputs must equal those of one
    # device-pointer call on the same inputs, bit for bit
    import torch
    nside, lmax, nt = 32, 64, 7
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    nc = 1 if spin == 0 else 2
    npix, nalm = 12 * nside * nside, sb.nalm_triangular(lmax)
    rng = np.random.default_rng(spin + 10 * jtype)

    def pinned(n, dtype):
        return torch.empty(n, dtype=dtype, pin_memory=True).numpy()

    if jtype == sb.SHARP_ALM2MAP:
        ins = [pinned(nalm, torch.complex128) for _ in range(nt * nc)]
        for i, x in enumerate(ins):
            x[:] = uniform_alm(lmax, seed=90 + i, spin=spin)
        outs = [pinned(npix, torch.float64) for _ in range(nt * nc)]
        for x in outs:
            x[:] = 0.0
        sb.execute(jtype, spin, ins, outs, g, a, nt, flags)
        d_in = [torch.view_as_real(torch.from_numpy(x.copy()).cuda()).reshape(-1) for x in ins]
        d_out = [torch.zeros(npix, dtype=torch.float64, device="cuda") for _ in outs]
        sb.execute_device(jtype, spin, d_in, d_out, g, a, nt, flags)
    else:
        ins = [pinned(npix, torch.float64) for _ in range(nt * nc)]
        for x in ins:
            x[:] = rng.standard_normal(npix)
        outs = [pinned(nalm, torch.complex128) for _ in range(nt * nc)]
        for x in outs:
            x[:] = 0.0
        sb.execute(jtype, spin, outs, ins, g, a, nt, flags)
        d_in = [torch.from_numpy(x.copy()).cuda() for x in ins]
        d_out = [torch.zeros(2 * nalm, dtype=torch.float64, device="cuda") for _ in outs]
        sb.execute_device(jtype, spin, d_out, d_in, g, a, nt, flags)
    torch.cuda.synchronize()
    for h, d in zip(outs, d_out):
        got = d.cpu().numpy()
        want = h.view(np.float64) if h.dtype == np.complex128 else h
        assert np.array_equal(got, want)


def test_workspace_stays_mapped_until_release_cache():
    # workspace comes from the library's own pool, which keeps it mapped
    # across synchronizes (a transform after a synchronize does not map it
    # again); sharp_b200_release_cache() hands it back to the driver.  The
    # results do not depend on whether the workspace was reused.
    import torch
    nside, lmax, nt = 512, 1024, 8
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    alms = [uniform_alm(lmax, seed=200 + i) for i in range(nt)]

    def run():
        maps = [np.zeros(12 * nside * nside) for _ in range(nt)]
        sb.execute(sb.SHARP_ALM2MAP, 0, [x.copy() for x in alms], maps, g, a, nt, DP | MIXED)
        return maps

    torch.cuda.synchronize()
    sb.lib().sharp_b200_release_cache()
    free0 = torch.cuda.mem_get_info()[0]
    first = run()
    torch.cuda.synchronize()
    reserved, used = sb.workspace_bytes()
    free1 = torch.cuda.mem_get_info()[0]
    second = run()                       # reuses the mapped workspace
    assert sb.workspace_bytes()[0] == reserved
    sb.lib().sharp_b200_release_cache()
    free2 = torch.cuda.mem_get_info()[0]
    print(f"workspace reserved {reserved} used {used}; free {free0} {free1} {free2}")
    # the phase array of one 4-transform piece is 2 (mmax+1) npairs 4 16 bytes
    assert reserved >= 2 * (lmax + 1) * (2 * nside) * 4 * 16
    assert used <= reserved
    assert free0 - free1 >= reserved - (64 << 20)      # held across the synchronize
    assert free2 - free1 >= reserved - (64 << 20)      # and handed back
    for x, y in zip(first, second):
        assert np.array_equal(x, y)
