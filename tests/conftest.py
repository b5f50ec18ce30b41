import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("planck-levels_b200", "oracle", "tests"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


# Library errors raise sharp_b200.SharpError inside the test session instead of
# ending the process (the reference's default, kept by the library).
os.environ.setdefault("SHARP_B200_ABORT_ON_ERROR", "0")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
