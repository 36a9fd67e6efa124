import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ppopp27-brdc-ae_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def built_lib():
    import build as brdc_build

    brdc_build.build()
    return brdc_build.LIB


@pytest.fixture(scope="session")
def solver(built_lib):
    import brdc

    s = brdc.Solver()
    yield s
    s.close()
