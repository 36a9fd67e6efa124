"""The reciprocal of the pole-root pair loops (brdc_rcp: hardware estimate
plus one third-order refinement step) against IEEE division on the device, over
magnitudes from 1e-300 to 1e300 and both signs, including powers of two
and their neighbours."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "ppopp27-brdc-ae_b200", "csrc")


def probe_lib() -> str:
    import build as brdc_build

    return brdc_build.nvcc_shared(os.path.join(HERE, "rcp_ulps.cu"),
                                  os.path.join(HERE, "librcp_ulps.so"),
                                  deps=[os.path.join(CSRC, "brdc_secular.cuh")], includes=[CSRC])


def ulps(x):
    lib = ctypes.CDLL(probe_lib())
    lib.brdc_probe_rcp_ulps.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    st = lib.brdc_probe_rcp_ulps(x.ctypes.data, out.ctypes.data, x.size)
    assert st == 0
    return out


def test_rcp_within_one_ulp(built_lib):
    rng = np.random.default_rng(0)
    mant = rng.uniform(1.0, 2.0, 1 << 20)
    expo = rng.integers(-990, 990, 1 << 20)
    x = np.ldexp(mant, expo) * rng.choice([-1.0, 1.0], 1 << 20)
    p2 = np.ldexp(1.0, np.arange(-990, 990))
    edges = np.concatenate([p2, np.nextafter(p2, 0), np.nextafter(p2, np.inf), -p2])
    u = ulps(np.concatenate([x, edges]))
    assert np.all(np.isfinite(u))
    assert u.max() <= 1.0, u.max()
    # almost always the correctly rounded value
    assert np.mean(u == 0.0) > 0.99
