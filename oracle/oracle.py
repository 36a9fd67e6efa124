"""Oracle loader -- TEST INFRASTRUCTURE ONLY.

ctypes bindings for ``liboracle.so``, the C restatement of the reference's
CPU boundary-row solver ``DSTEDC_DC_BR`` (cpu/src/dstedc_dc_br.f:7) and its
helpers, plus the LAPACK baselines the reference compares against
(DSTERF: scripts/cpu/smoke_br.f90:30; DSTEDC('N'):
gpu/bench/tridiag_dc_bench.cu:868-907).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, always as the checker or as the timed CPU
reference; the product path never does.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def lapack_path() -> str:
    """Path of scipy's bundled OpenBLAS, which provides the LAPACK routines
    (DLAED4, DSTEQR, DSTERF, ...) the reference links against."""
    import scipy

    libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libs, "libscipy_openblas*.so*")))
    if not cands:
        raise RuntimeError("scipy's OpenBLAS (LAPACK provider) not found under " + libs)
    return cands[0]


def build() -> None:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
        os.path.join(_HERE, "brdc_oracle.c")
    ):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    lib.oracle_init.argtypes = [ctypes.c_char_p]
    lib.oracle_init.restype = ctypes.c_int
    rc = lib.oracle_init(lapack_path().encode())
    if rc != 0:
        raise RuntimeError(f"oracle_init failed ({rc})")
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    lib.oracle_dstedc_dc_br.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, ip, ctypes.c_int]
    lib.oracle_dstedc_dc_br.restype = ctypes.c_int
    lib.oracle_solve.argtypes = [ctypes.c_int, dp, dp, ip, ctypes.c_int, ip]
    lib.oracle_solve.restype = ctypes.c_int
    lib.oracle_dsterf.argtypes = [ctypes.c_int, dp, dp]
    lib.oracle_dsterf.restype = ctypes.c_int
    lib.oracle_dstedc_n.argtypes = [ctypes.c_int, dp, dp]
    lib.oracle_dstedc_n.restype = ctypes.c_int
    lib.oracle_dlaed4.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, ctypes.c_double, dp]
    lib.oracle_dlaed4.restype = ctypes.c_int
    lib.oracle_max_threads.restype = ctypes.c_int
    lib.oracle_set_threads.argtypes = [ctypes.c_int]
    lib.brdc_wprod_nthreads.restype = ctypes.c_int
    _lib = lib
    return lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def set_threads(nt: int) -> None:
    _load().oracle_set_threads(int(nt))


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def dstedc_dc_br_query(n: int) -> tuple[int, int]:
    """LWORK=-1 query: (LWMIN, LIWMIN) as DSTEDC_DC_BR reports them."""
    lib = _load()
    w = np.zeros(1)
    iw = np.zeros(1, dtype=np.int32)
    info = lib.oracle_dstedc_dc_br(int(n), _dp(np.zeros(1)), _dp(np.zeros(1)), _dp(w), -1, _ip(iw), -1)
    if info != 0:
        raise ValueError(f"DSTEDC_DC_BR query INFO={info}")
    return int(w[0]), int(iw[0])


def dstedc_dc_br(d, e, return_kdefl: bool = False):
    """Eigenvalues (ascending) of the symmetric tridiagonal (d, e) by the
    restated DSTEDC_DC_BR.  With ``return_kdefl`` also returns K of every
    merge in execution order.  Raises on INFO != 0."""
    lib = _load()
    d = np.array(d, dtype=np.float64, copy=True)
    n = d.shape[0]
    e = np.array(e, dtype=np.float64, copy=True)
    if e.shape[0] < max(n - 1, 0):
        raise ValueError("e must hold n-1 entries")
    e = np.concatenate([e[: max(n - 1, 0)], np.zeros(1)])
    cap = max(n, 1)
    kd = np.full(cap, -1, dtype=np.int32)
    kl = np.zeros(1, dtype=np.int32)
    info = lib.oracle_solve(n, _dp(d), _dp(e), _ip(kd), cap, _ip(kl))
    if info != 0:
        raise RuntimeError(f"DSTEDC_DC_BR INFO={info}")
    if return_kdefl:
        return d, kd[: int(kl[0])].copy()
    return d


def dsterf(d, e) -> np.ndarray:
    lib = _load()
    d = np.array(d, dtype=np.float64, copy=True)
    n = d.shape[0]
    e = np.concatenate([np.array(e, dtype=np.float64)[: max(n - 1, 0)], np.zeros(1)])
    info = lib.oracle_dsterf(n, _dp(d), _dp(e))
    if info != 0:
        raise RuntimeError(f"DSTERF INFO={info}")
    return d


def dstedc_n(d, e) -> np.ndarray:
    lib = _load()
    d = np.array(d, dtype=np.float64, copy=True)
    n = d.shape[0]
    e = np.concatenate([np.array(e, dtype=np.float64)[: max(n - 1, 0)], np.zeros(1)])
    info = lib.oracle_dstedc_n(n, _dp(d), _dp(e))
    if info != 0:
        raise RuntimeError(f"DSTEDC INFO={info}")
    return np.sort(d)


def dlaed4(d, z, rho: float, i: int):
    """LAPACK DLAED4 for root ``i`` (0-based): returns (lambda, delta)."""
    lib = _load()
    d = np.ascontiguousarray(d, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.float64)
    delta = np.zeros_like(d)
    lam = np.zeros(1)
    info = lib.oracle_dlaed4(d.shape[0], int(i) + 1, _dp(d), _dp(z), _dp(delta), float(rho), _dp(lam))
    if info != 0:
        raise RuntimeError(f"DLAED4 INFO={info}")
    return float(lam[0]), delta
