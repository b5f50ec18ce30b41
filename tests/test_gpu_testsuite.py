"""The reference's own C test program (libsharp/sharp_testsuite.c, built by
oracle/Makefile against the reference headers and linked against
libsharp_b200.so in place of libsharp) run on the GPU: a compiled C caller
of the drop-in, unchanged.

* acctest: the 18 known answers of check_sign_scale (sharp_testsuite.c:
  337-443, relative 1e-12) and round trips on a Gauss grid, lmax 127,
  spins 0/1/2/3/30, ntrans 1..6, every nv hint, error < 1e-10 (:490-529);
* test: the timed round trip on a Gauss grid (exact quadrature, so the
  reported errors must be at round-off level) and on the HEALPix grid."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "sharp_testsuite_b200")


def _run(*args, timeout=600):
    if not os.path.exists(EXE):
        pytest.skip("sharp_testsuite_b200 not built (make -C oracle)")
    env = dict(os.environ, SHARP_B200_ABORT_ON_ERROR="1", OMP_NUM_THREADS="1")
    r = subprocess.run([EXE, *args], capture_output=True, text=True, timeout=timeout, env=env)
    print(r.stdout[-3000:])
    print(r.stderr[-2000:])
    return r


def test_reference_acctest_through_the_drop_in():
    r = _run("acctest")
    assert r.returncode == 0
    assert r.stdout.count("Passed.") == 2


@pytest.mark.parametrize("args,bound", [
    (("gauss", "1023", "-1", "-1", "-1", "2", "4"), 1e-10),
    (("gauss", "2047", "-1", "-1", "-1", "0", "1"), 1e-10),
    (("healpix", "1024", "-1", "512", "-1", "2", "1"), None)])
def test_reference_timed_test_through_the_drop_in(args, bound):
    r = _run("test", *args)
    assert r.returncode == 0
    assert "wall time for alm2map" in r.stdout and "wall time for map2alm" in r.stdout
    errs = [float(x) for x in re.findall(r"component \d+: rms ([0-9.eE+-]+)", r.stdout)]
    assert errs
    if bound is not None:
        assert max(errs) < bound
