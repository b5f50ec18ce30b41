"""Generates tests/golden/reference_small.npz from the reference libsharp
(compiled by oracle/Makefile from the zonca/planck-levelS sources).

Run in a checkout where oracle/_ref/libsharp_ref.so exists:
    python tests/golden/make_golden.py
Each case stores its seeded inputs and the reference outputs, so the tests
need neither the reference sources nor its library to check the oracle and
the GPU engine against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import ref  # noqa: E402
from helpers import random_alm, uniform_alm  # noqa: E402

DP = 1 << 4
CASES = [
    # name, geometry, lmax, mmax, spin, jtype
    ("hpx16_l32_s0", ("healpix", 16), 32, 32, 0, 1),
    ("hpx16_l32_s2", ("healpix", 16), 32, 32, 2, 1),
    ("hpx8_l40_m20_s0_alias", ("healpix", 8), 40, 20, 0, 1),
    ("gauss_l24_s1_deriv", ("gauss", 25, 50), 24, 24, 1, 4),
    ("gauss_l24_s3", ("gauss", 25, 49), 24, 24, 3, 1),
]


def geometry(spec):
    if spec[0] == "healpix":
        return ref.healpix(spec[1])
    return ref.grid(spec[0], spec[1], spec[2])


def main():
    out = {}
    for name, gspec, lmax, mmax, spin, jtype in CASES:
        g = geometry(gspec)
        a = ref.triangular(lmax, mmax)
        npix = g.npix()
        nalm = 1 if (spin == 0 or jtype == 4) else 2
        nmaps = 1 if (spin == 0 and jtype == 1) else 2
        alms = [random_alm(lmax, mmax, seed=100 + i) if spin == 0 else
                uniform_alm(lmax, mmax, seed=100 + i, spin=spin) for i in range(nalm)]
        maps = [np.zeros(npix) for _ in range(nmaps)]
        ref.execute(jtype, spin, [x.copy() for x in alms], maps, g, a, 1, DP)
        back = [np.zeros_like(alms[0]) for _ in range(nalm)]
        if jtype == 1:
            ref.execute(0, spin, back, [m.copy() for m in maps], g, a, 1, DP)
        for i in range(nalm):
            out[f"{name}/alm{i}"] = alms[i]
            out[f"{name}/back{i}"] = back[i]
        for i in range(nmaps):
            out[f"{name}/map{i}"] = maps[i]
    np.savez_compressed(os.path.join(HERE, "reference_small.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
