"""The solver under its LAPACK names (dstebr_, sstebr_, LAPACKE_dstebr,
LAPACKE_sstebr and their _work forms): host arrays in, ascending eigenvalues
out, against the oracle and LAPACK DSTERF."""
import ctypes

import numpy as np
import pytest

import oracle
from brdc import families

pytestmark = pytest.mark.gpu
TOL = 1e-12  # max |lambda - lambda_ref| / ||T||_2 (FP64 entries)


def _lib(built_lib):
    lib = ctypes.CDLL(built_lib)
    for name in ("LAPACKE_dstebr", "LAPACKE_sstebr", "LAPACKE_dstebr_work", "LAPACKE_sstebr_work"):
        getattr(lib, name).restype = ctypes.c_int
    return lib


def rel_err(w, ref):
    return float(np.max(np.abs(np.asarray(w, dtype=np.float64) - ref)) / np.max(np.abs(ref)))


def fortran_call(fn, d, e, dtype):
    n = len(d)
    ci = ctypes.c_int
    D = np.array(d, dtype=dtype)
    E = np.array(e if n > 1 else [0.0], dtype=dtype)
    wq, iwq, info = np.zeros(1, dtype=dtype), np.zeros(1, dtype=np.int32), ci(0)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    fn(ctypes.byref(ci(n)), P(D), P(E), P(wq), ctypes.byref(ci(-1)), P(iwq), ctypes.byref(ci(-1)),
       ctypes.byref(info))
    assert info.value == 0
    lw, liw = int(wq[0]), int(iwq[0])
    work, iwork = np.zeros(lw, dtype=dtype), np.zeros(liw, dtype=np.int32)
    fn(ctypes.byref(ci(n)), P(D), P(E), P(work), ctypes.byref(ci(lw)), P(iwork), ctypes.byref(ci(liw)),
       ctypes.byref(info))
    return info.value, D


@pytest.mark.parametrize("n", [2, 26, 1000, 5000])
def test_dstebr_fortran(built_lib, n):
    d, e = families.generate("normal", n)
    info, w = fortran_call(_lib(built_lib).dstebr_, d, e, np.float64)
    assert info == 0
    assert np.all(np.diff(w) >= 0)
    assert rel_err(w, oracle.dstedc_dc_br(d, e)) < TOL
    assert rel_err(w, np.sort(oracle.dsterf(d, e))) < TOL


@pytest.mark.parametrize("n", [2, 26, 3000])
def test_sstebr_fortran(built_lib, n):
    d, e = families.generate("uniform", n)
    df, ef = d.astype(np.float32), e.astype(np.float32)
    info, w = fortran_call(_lib(built_lib).sstebr_, df, ef, np.float32)
    assert info == 0 and w.dtype == np.float32
    # FP64 eigenvalues of the float matrix, rounded once to float
    ref = np.sort(oracle.dsterf(df.astype(np.float64), ef.astype(np.float64)))
    assert rel_err(w, ref) <= 2.0 ** -23


def test_lapacke_forms(built_lib):
    lib = _lib(built_lib)
    n = 4096
    d, e = families.generate("clustered", n)
    ref = np.sort(oracle.dsterf(d, e))
    D, E = d.copy(), e.copy()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.LAPACKE_dstebr(n, P(D), P(E)) == 0
    assert rel_err(D, ref) < TOL
    # _work form with the caller's workspace, sized by its query
    wq, iwq = np.zeros(1), np.zeros(1, dtype=np.int32)
    assert lib.LAPACKE_dstebr_work(n, P(d.copy()), P(e.copy()), P(wq), -1, P(iwq), -1) == 0
    lw = int(wq[0])
    assert lw >= 18 * n and int(iwq[0]) == 7 * n
    work, iwork = np.zeros(lw), np.zeros(7 * n, dtype=np.int32)
    D2, E2 = d.copy(), e.copy()
    assert lib.LAPACKE_dstebr_work(n, P(D2), P(E2), P(work), lw, P(iwork), 7 * n) == 0
    assert np.array_equal(D, D2)
    # too small a workspace: INFO = -5 from the routine, D untouched
    D3 = d.copy()
    assert lib.LAPACKE_dstebr_work(n, P(D3), P(e.copy()), P(work), 10, P(iwork), 7 * n) == -5
    assert np.array_equal(D3, d)
    df, ef = d.astype(np.float32), e.astype(np.float32)
    assert lib.LAPACKE_sstebr(n, P(df), P(ef)) == 0
    reff = np.sort(oracle.dsterf(d.astype(np.float32).astype(np.float64),
                                 e.astype(np.float32).astype(np.float64)))
    assert rel_err(df, reff) <= 2.0 ** -23
