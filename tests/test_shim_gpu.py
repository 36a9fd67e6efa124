"""The evd::internal forwarding shim driven as the reference's bench drives
its solver: same results as the C ABI, and the reference's argument checks
(gpu/src/tridiag_solver.cu:2545-2557): uplo other than LOWER, the CPU
backend, or AUTO with n < 17 give EVD_STATUS_INVALID_VALUE."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from brdc import families

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM_LIB = os.path.join(HERE, "libshim_check.so")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(SHIM_LIB), reason="shim not built")]
AUTO, CPU, GPU = 0, 1, 2
LOWER, UPPER = 0, 1


@pytest.fixture(scope="module")
def shim(solver):
    lib = ctypes.CDLL(SHIM_LIB)
    vp = ctypes.c_void_p
    lib.shim_workspace_size.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_size_t)]
    lib.shim_solve.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp,
                               vp, vp, ctypes.c_size_t, vp]
    return lib


def run(shim, d, e, uplo=LOWER, backend=GPU, vectors=0):
    import torch

    n = len(d)
    nb = ctypes.c_size_t()
    assert shim.shim_workspace_size(n, ctypes.byref(nb)) == 0
    ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e if len(e) else np.zeros(1), device="cuda")
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    st = shim.shim_solve(n, uplo, backend, vectors, D.data_ptr(), E.data_ptr(), W.data_ptr(),
                         ws.data_ptr(), nb.value, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return st, W.cpu().numpy()


@pytest.mark.parametrize("n", [17, 1000, 16384])
def test_shim_solves_like_the_library(shim, n):
    d, e = families.generate("normal", n)
    st, w = run(shim, d, e)
    assert st == 0
    ref = oracle.dstedc_dc_br(d, e)
    assert np.max(np.abs(w - ref)) < 1e-12 * np.max(np.abs(ref))


def test_shim_argument_checks(shim):
    d, e = families.generate("normal", 100)
    assert run(shim, d, e, uplo=UPPER)[0] == 3
    assert run(shim, d, e, backend=CPU)[0] == 3
    assert run(shim, d, e, backend=AUTO)[0] == 0
    d16, e16 = families.generate("normal", 16)
    assert run(shim, d16, e16, backend=AUTO)[0] == 3
    assert run(shim, d16, e16, backend=GPU)[0] == 0
    assert run(shim, d, e, vectors=1)[0] == 8
