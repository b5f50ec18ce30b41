"""The FP64 pass-width tuner (the counterpart of the reference's nv oracle):
it runs on the first job of a shape with several transforms, not for single
transforms, not when the flags carry a vector-count hint (SHARP_NVMAX bits),
and its decision leaves the results bit-identical to single-transform jobs.
Each case runs in a fresh process (the decisions are kept per process)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

SCRIPT = r'''
import sys
sys.path.insert(0, {pkg!r})
import numpy as np
import sharp_b200 as sb
nside, lmax, nt, hint = 32, 64, {nt}, {hint}
g, a = sb.Geometry.healpix(nside), sb.AlmInfo.triangular(lmax)
rng = np.random.default_rng(1)
nalm = sb.nalm_triangular(lmax)
alms = [rng.standard_normal(nalm) + 1j * rng.standard_normal(nalm) for _ in range(nt)]
for x in alms:
    x[:lmax + 1] = x[:lmax + 1].real
maps = [np.zeros(12 * nside * nside) for _ in range(nt)]
sb.execute(sb.SHARP_ALM2MAP, 0, [x.copy() for x in alms], maps, g, a, nt, sb.SHARP_DP | hint)
back = [np.zeros(nalm, np.complex128) for _ in range(nt)]
sb.execute(sb.SHARP_MAP2ALM, 0, back, [m.copy() for m in maps], g, a, nt, sb.SHARP_DP | hint)
for i in range(nt):
    m1 = [np.zeros(12 * nside * nside)]
    sb.execute(sb.SHARP_ALM2MAP, 0, [alms[i].copy()], m1, g, a, 1, sb.SHARP_DP)
    b1 = [np.zeros(nalm, np.complex128)]
    sb.execute(sb.SHARP_MAP2ALM, 0, b1, [maps[i].copy()], g, a, 1, sb.SHARP_DP)
    assert np.array_equal(m1[0], maps[i]) and np.array_equal(b1[0], back[i])
print("ok")
'''


def _run(nt, hint):
    env = dict(os.environ, SHARP_B200_TUNE_LOG="1")
    env.pop("SHARP_B200_TUNE", None)
    code = SCRIPT.format(pkg=os.path.join(ROOT, "planck-levels_b200"), nt=nt, hint=hint)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().endswith("ok")
    return [l for l in r.stderr.splitlines() if l.startswith("sharp_b200 tuner:")]


def test_tuner_decides_once_per_direction_for_several_transforms():
    lines = _run(4, 0)
    assert len(lines) == 2, lines
    assert "synthesis" in lines[0] and "analysis" in lines[1]
    assert all("width 1" in l and "width 2" in l and "width 4" in l for l in lines)


def test_tuner_skips_single_transforms_and_vector_count_hints():
    assert _run(1, 0) == []
    assert _run(4, 3) == []      # nv hint in the SHARP_NVMAX bits
