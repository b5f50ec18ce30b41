"""One transform over several GPUs: one process per GPU (torch.distributed
with NCCL), the ring pairs of the geometry split between the ranks.

The reference scales a transform over MPI tasks with sharp_execute_mpi
(libsharp/sharp_mpi.c:210-327): each task takes a set of m values for the
Legendre step and a set of rings for the FFT, and MPI_Alltoallv transposes
the phase array between the two steps (2 ntrans nmaps (mmax+1) complex values
per ring pair cross the network in each direction).  Here both steps are split
by ring pair instead: a pair's Legendre work (every m up to its mlim) and its
ring FFTs stay on the GPU that owns it.  Synthesis then needs no
communication, and analysis needs one all-reduce of the partial a_lm (summed
in the NVLink switch where NCCL uses NVLS).  At Nside 2048 / lmax 4096 that is
134 MB per component instead of the 537 MB of phase the transpose moves, and
the reduction runs once at the end instead of between the two steps.

Pairs are assigned by a greedy longest-processing-time rule on their cost
(Legendre (l, m) terms plus ring FFT work), which balances the ranks to well
under 1% on HEALPix grids.

Each rank calls ``execute`` with the full geometry, the full a_lm layout and
full-size arrays:

* alm2map / WY / DERIV1: the rank's maps get the pixels of its own rings (the
  reference's tasks likewise hold only their local rings); gather=True sums
  the maps over the ranks so that every rank holds the whole map.
* map2alm / Yt: every rank's a_lm outputs hold the complete result.

SHARP_ADD and SHARP_SUBTRACT keep their meaning for the complete result.
Because outputs are summed over the ranks, every entry of the summed arrays
must belong to the layout: a_lm arrays exactly the extent of their layout
(triangular or rectangular with unit stride, as Alm<T> keeps them) and, with
gather=True, maps whose pixels are all on rings of the geometry.
"""
from __future__ import annotations

import math

import numpy as np

from . import (SHARP_ADD, SHARP_ADJOINT, SHARP_ALM2MAP, SHARP_MAP2ALM, SHARP_SUBTRACT,
               SHARP_WY, SHARP_Yt, lib)

_ADJ = {0: SHARP_WY, 1: SHARP_Yt, 2: SHARP_ALM2MAP, 3: SHARP_MAP2ALM}


def _pairs(geom):
    g = geom.ptr.contents
    return [g.pair[i] for i in range(g.npairs)]


def pair_costs(geom, lmax: int, mmax: int, spin: int) -> np.ndarray:
    """Work of each ring pair: its Legendre (l, m) terms (the same mlim rule as
    the transform) plus an FFT term of 8 n log2 n per ring."""
    get_mlim = lib().sharp_get_mlim
    out = []
    for pr in _pairs(geom):
        ml = min(get_mlim(lmax, spin, pr.r1.sth, pr.r1.cth), mmax)
        terms = 0
        if ml >= 0:
            m = np.arange(ml + 1)
            terms = int(np.maximum(lmax - np.maximum(m, spin) + 1, 0).sum())
        fft = sum(8.0 * n * math.log2(max(n, 2)) for n in (pr.r1.nph, pr.r2.nph) if n > 0)
        out.append(terms + fft)
    return np.asarray(out, np.float64)


def partition(costs, world: int) -> list:
    """Pair indices of each rank: greedy longest-processing-time assignment
    (deterministic: ties go to the lowest rank), each list in ascending
    order."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


class RingSplit:
    """This rank's share of a geometry: the pair indices and the geometry
    made of them.  ``subset(geom, pairs)`` builds that geometry (default:
    Geometry.subset of this library)."""

    def __init__(self, geom, lmax: int, mmax: int, spin: int, rank: int, world: int,
                 subset=None):
        self.world, self.rank, self.geom = world, rank, geom
        self.costs = pair_costs(geom, lmax, mmax, spin)
        self.parts = partition(self.costs, world)
        self.pairs = self.parts[rank]
        self.local = (subset or (lambda g, p: g.subset(p)))(geom, self.pairs)

    def imbalance(self) -> float:
        """Largest rank load over the mean load, minus one."""
        loads = [float(self.costs[p].sum()) for p in self.parts]
        return max(loads) / (sum(loads) / len(loads)) - 1.0


def _entries(x) -> int:
    n = x.size if isinstance(x, np.ndarray) else x.numel()
    real = (x.dtype.kind != "c") if isinstance(x, np.ndarray) else not x.is_complex()
    return n // 2 if real else n       # complex entries (a_lm given as float64 views)


def _check_dense(alm_arrays, ainfo, map_arrays, geom, need_alm, need_maps):
    if need_alm:
        a = ainfo.ptr.contents
        nent = sum(a.lmax - a.mval[i] + 1 for i in range(a.nm))
        if a.stride != 1 or a.flags != 0 or any(_entries(x) != nent for x in alm_arrays):
            raise ValueError("the a_lm arrays must hold exactly their layout's entries "
                             "(unit stride, no gaps) to be summed over the ranks")
    if need_maps:
        npix = geom.npix()
        for x in map_arrays:
            n = x.size if isinstance(x, np.ndarray) else x.numel()
            if n != npix:
                raise ValueError("gather=True needs maps whose pixels are all on rings")


def _zeros_like(x):
    if isinstance(x, np.ndarray):
        return np.zeros_like(x)
    import torch
    return torch.zeros_like(x)


def _torch_all_reduce(arrays, group=None):
    import torch
    import torch.distributed as dist
    for x in arrays:
        t = x
        if isinstance(x, np.ndarray):
            t = torch.from_numpy(x.view(np.float64) if x.dtype.kind == "c" else x)
        elif t.is_complex():
            t = torch.view_as_real(t)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def execute(split: RingSplit, jtype: int, spin: int, alm, maps, ainfo, ntrans: int, flags: int,
            run=None, all_reduce=None, gather: bool = False, group=None):
    """One rank's part of a transform split by ring pairs (see the module
    text).  ``run(jtype, spin, alm, maps, geom, ainfo, ntrans, flags)`` runs
    a transform on this rank's GPU (default: sharp_b200.execute_device on
    CUDA tensors); ``all_reduce(list of arrays)`` sums arrays over the ranks
    in place (default: torch.distributed.all_reduce).  Every rank makes the
    same collective calls in the same order."""
    if run is None:
        from . import execute_device as run
    if all_reduce is None:
        def all_reduce(xs):
            _torch_all_reduce(xs, group)
    eff = _ADJ[jtype] if (flags & SHARP_ADJOINT) and jtype in _ADJ else jtype
    outputs_alm = eff in (SHARP_MAP2ALM, SHARP_Yt)
    _check_dense(alm, ainfo, maps, split.geom, outputs_alm, gather and not outputs_alm)
    acc = flags & (SHARP_ADD | SHARP_SUBTRACT)
    base = flags & ~(SHARP_ADD | SHARP_SUBTRACT)
    if outputs_alm or gather:
        outs = alm if outputs_alm else maps
        if acc:
            # the partial results of all ranks are summed first, then added
            tmp = [_zeros_like(x) for x in outs]
            if outputs_alm:
                run(jtype, spin, tmp, maps, split.local, ainfo, ntrans, base)
            else:
                run(jtype, spin, alm, tmp, split.local, ainfo, ntrans, base)
            all_reduce(tmp)
            for x, t in zip(outs, tmp):
                if acc & SHARP_ADD:
                    x += t
                else:
                    x -= t
        else:
            if not outputs_alm:
                # pixels of the other ranks' rings must be zero before the sum
                for x in outs:
                    x[...] = 0
            run(jtype, spin, alm, maps, split.local, ainfo, ntrans, base)
            all_reduce(outs)
    else:
        run(jtype, spin, alm, maps, split.local, ainfo, ntrans, flags)
