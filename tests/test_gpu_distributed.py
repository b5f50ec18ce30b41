"""The per-GPU part of a transform split over several GPUs by ring pairs
(sharp_b200.distributed), on one GPU: every rank's share runs here in turn
through the C ABI on its subset geometry (sharp_b200_make_subset_geom_info).
The synthesis of each share must reproduce the full transform's pixels on
its rings, and the partial analyses must sum to the full a_lm, FP64 within
1e-12 and SHARP_MIXED within 1e-6 of the full FP64 transform.  The
collective that sums the partial a_lm across processes is tested with gloo
ranks on the CPU (test_dist_cpu.py); this run has one GPU."""
import numpy as np
import pytest

import sharp_b200 as sb
from helpers import rel_l2, uniform_alm

pytestmark = pytest.mark.gpu
DP, MIXED = sb.SHARP_DP, sb.SHARP_MIXED


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("spin", [0, 2])
@pytest.mark.parametrize("flags,tol", [(DP, 1e-12), (DP | MIXED, 1e-6)])
def test_ring_shares_reproduce_the_full_transform(world, spin, flags, tol):
    import torch
    from sharp_b200 import distributed as sd
    nside, lmax = 128, 256
    g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
    npix, nalm = 12 * nside * nside, sb.nalm_triangular(lmax)
    nc = 1 if spin == 0 else 2
    dev = "cuda"
    alms = [torch.from_numpy(uniform_alm(lmax, seed=50 + i, spin=spin)).to(dev) for i in range(nc)]
    va = [torch.view_as_real(x).reshape(-1) for x in alms]
    full = [torch.zeros(npix, dtype=torch.float64, device=dev) for _ in range(nc)]
    sb.execute_device(sb.SHARP_ALM2MAP, spin, va, full, g, a, 1, DP)
    want = [torch.zeros(2 * nalm, dtype=torch.float64, device=dev) for _ in range(nc)]
    sb.execute_device(sb.SHARP_MAP2ALM, spin, want, full, g, a, 1, DP)
    total = [torch.zeros_like(x) for x in want]
    covered = torch.zeros(npix, dtype=torch.int32, device=dev)
    splits = [sd.RingSplit(g, lmax, lmax, spin, r, world) for r in range(world)]
    assert sorted(i for s in splits for i in s.pairs) == list(range(g.npairs))
    for s in splits:
        assert s.imbalance() < 0.02
        mine = [torch.zeros(npix, dtype=torch.float64, device=dev) for _ in range(nc)]
        sb.execute_device(sb.SHARP_ALM2MAP, spin, va, mine, s.local, a, 1, flags)
        gi = s.local.ptr.contents
        idx = torch.from_numpy(np.concatenate(
            [r.ofs + np.arange(r.nph) for i in range(gi.npairs)
             for r in (gi.pair[i].r1, gi.pair[i].r2) if r.nph > 0])).to(dev)
        covered[idx] += 1
        for x, y in zip(mine, full):
            assert rel_l2(x[idx].cpu().numpy(), y[idx].cpu().numpy()) < tol
        part = [torch.zeros_like(x) for x in want]
        sb.execute_device(sb.SHARP_MAP2ALM, spin, part, full, s.local, a, 1, flags)
        for t, p in zip(total, part):
            t += p
    torch.cuda.synchronize()
    assert bool((covered == 1).all())          # every pixel on exactly one rank
    for x, y in zip(total, want):
        assert rel_l2(x.cpu().numpy(), y.cpu().numpy()) < tol
