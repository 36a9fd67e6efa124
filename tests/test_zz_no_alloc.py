"""The allocation-free entry point brdc_dstebr_noalloc, called through the
C ABI, against the workspace entry brdc_dstebr.

It exists for callers that cannot allocate device memory when they solve
(host callbacks and stream-ordered sections where cudaMalloc is not
allowed, plug-ins whose host owns every allocation); its scratch is a
static device array inside the library.  This file is collected last so a
failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

import brdc
import oracle
from brdc import families

pytestmark = pytest.mark.gpu
TOL = 1e-12  # max |lambda - lambda_ref| / ||T||_2, as in the other parity tests


def test_noalloc_matches_workspace_entry_twice(solver):
    """Two calls in a row, each against the workspace entry and against the
    oracle (the C restatement of the reference's DSTEDC_DC_BR); the status
    word the solve left in the static array reads 0."""
    import torch

    lib = brdc.load()
    for family, n in (("normal", 5000), ("uniform", 16384)):
        d, e = families.generate(family, n)
        D = torch.tensor(d, device="cuda")
        E = torch.tensor(e, device="cuda")
        ref = solver.dstebr(D, E).cpu().numpy()
        W = torch.empty(n, dtype=torch.float64, device="cuda")
        st = lib.brdc_dstebr_noalloc(solver.h, n, ctypes.c_void_p(D.data_ptr()),
                                     ctypes.c_void_p(E.data_ptr()), ctypes.c_void_p(W.data_ptr()))
        assert st == brdc.SUCCESS
        w = W.cpu().numpy()
        assert np.max(np.abs(w - ref)) <= TOL * np.max(np.abs(ref))
        orc = oracle.dstedc_dc_br(d, e)
        assert np.max(np.abs(w - orc)) <= TOL * np.max(np.abs(orc))
        assert solver.noalloc_info_status() == (0, brdc.SUCCESS)


def test_noalloc_status_reports_non_finite_input(solver):
    import torch

    n = 2000
    d, e = families.generate("normal", n)
    d[7] = np.nan
    solver.dstebr_noalloc(torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda"))
    assert solver.noalloc_info_status() == (-4, brdc.INTERNAL_ERROR)
    d[7] = 0.5
    W = solver.dstebr_noalloc(torch.tensor(d, device="cuda"),
                              torch.tensor(e, device="cuda")).cpu().numpy()
    assert solver.noalloc_info_status() == (0, brdc.SUCCESS)
    orc = oracle.dstedc_dc_br(d, e)
    assert np.max(np.abs(W - orc)) <= TOL * np.max(np.abs(orc))


def test_noalloc_rejects_orders_beyond_its_scratch(solver):
    import torch

    n = 16385
    D = torch.zeros(n, dtype=torch.float64, device="cuda")
    E = torch.zeros(n, dtype=torch.float64, device="cuda")
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    st = brdc.load().brdc_dstebr_noalloc(solver.h, n, ctypes.c_void_p(D.data_ptr()),
                                         ctypes.c_void_p(E.data_ptr()), ctypes.c_void_p(W.data_ptr()))
    assert st == brdc.INVALID_VALUE
