import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libgg.so")
    config.addinivalue_line("markers", "ref: needs the reference build under oracle/_ref")


def _ensure_oracle():
    for lib, src in (("liboracle.so", "oracle.c"), ("liboracle_fm.so", "fm_draws.cc")):
        lib, src = os.path.join(ROOT, "oracle", lib), os.path.join(ROOT, "oracle", src)
        if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


_ensure_oracle()


@pytest.fixture(scope="session")
def ctx():
    from graptor_b200 import gg
    c = gg.Context(0)
    yield c
    c.close()
