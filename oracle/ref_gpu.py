"""Reference CUDA prototype wrapper -- TEST AND BENCHMARK INFRASTRUCTURE ONLY.

Loads ``oracle/_ref/libref_brdc_gpu.so`` (the reference's gpu/src sources
compiled for sm_100a by ``oracle/build_ref.sh``) and calls its values-only
solve entry ``tridiag_solver_run_from_device_tridiagonal``
(gpu/src/tridiag_solver.cu:2541) through the C shim in ``ref_shim.cu``.
Used as a checker (per-level deflation counts) and as the timed reference
CUDA baseline; the product never calls it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_brdc_gpu.so")
MERGE_LIB_PATH = os.path.join(_HERE, "_ref", "libref_merge.so")
_lib = None
_merge_lib = None


def merge_available() -> bool:
    return os.path.exists(MERGE_LIB_PATH)


def merge_level(child_sizes, D, E, first_rows, last_rows) -> dict:
    """The reference's own deflation kernels (ref_merge.cu) on one merge
    level: child_sizes [2 per merge], D, E, first_rows, last_rows by row.
    Returns mask0, mask, map, md, ndd, dcount, z, cc, ss, tol, rho."""
    global _merge_lib
    if _merge_lib is None:
        if not merge_available():
            raise RuntimeError("reference deflation kernels not built (oracle/build_ref.sh)")
        lib = ctypes.CDLL(MERGE_LIB_PATH)
        ip = ctypes.POINTER(ctypes.c_int)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.ref_merge_level.argtypes = [ctypes.c_int, ctypes.c_int, ip, dp, dp, dp, dp,
                                        ip, ip, ip, dp, ip, ip, dp, dp, dp, dp, dp]
        _merge_lib = lib
    cs = np.ascontiguousarray(child_sizes, dtype=np.int32)
    n = int(cs.sum())
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in (D, E, first_rows, last_rows)]
    out = {k: np.zeros(n, dtype=np.int32) for k in ("mask0", "mask", "map", "ndd", "dcount")}
    out.update({k: np.zeros(n) for k in ("md", "z", "cc", "ss", "tol", "rho")})
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    st = _merge_lib.ref_merge_level(
        n, len(cs) // 2, cs.ctypes.data_as(ip), *[a.ctypes.data_as(dp) for a in args],
        out["mask0"].ctypes.data_as(ip), out["mask"].ctypes.data_as(ip), out["map"].ctypes.data_as(ip),
        out["md"].ctypes.data_as(dp), out["ndd"].ctypes.data_as(ip), out["dcount"].ctypes.data_as(ip),
        out["z"].ctypes.data_as(dp), out["cc"].ctypes.data_as(dp), out["ss"].ctypes.data_as(dp),
        out["tol"].ctypes.data_as(dp), out["rho"].ctypes.data_as(dp))
    if st != 0:
        raise RuntimeError(f"ref_merge_level status {st}")
    return out


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise RuntimeError("reference prototype not built (oracle/build_ref.sh)")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    lib.ref_init.argtypes = [ctypes.c_char_p]
    lib.ref_create.argtypes = [ctypes.POINTER(vp)]
    lib.ref_destroy.argtypes = [vp]
    lib.ref_stream.argtypes = [vp]
    lib.ref_stream.restype = vp
    lib.ref_workspace_size.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_size_t)]
    lib.ref_solve.argtypes = [vp, ctypes.c_int64, vp, vp, vp, vp, ctypes.c_size_t, ctypes.c_int]
    lib.ref_level_diagnostics.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    try:
        import oracle

        lib.ref_init(oracle.lapack_path().encode())
    except Exception:
        lib.ref_init(None)
    _lib = lib
    return lib


def workspace_size(n: int) -> int:
    out = ctypes.c_size_t()
    st = _load().ref_workspace_size(int(n), ctypes.byref(out))
    if st != 0:
        raise RuntimeError(f"reference workspace query status {st}")
    return int(out.value)


class RefSolver:
    """The reference prototype on its own (non-blocking) handle stream."""

    def __init__(self):
        import torch

        self.torch = torch
        lib = _load()
        h = ctypes.c_void_p()
        st = lib.ref_create(ctypes.byref(h))
        if st != 0:
            raise RuntimeError(f"evd_create_handle status {st}")
        self.h = h
        self.stream = torch.cuda.ExternalStream(lib.ref_stream(h))
        self._ws = {}

    def close(self):
        if self.h:
            _load().ref_destroy(self.h)
            self.h = None

    def workspace(self, n):
        ws = self._ws.get(n)
        if ws is None:
            ws = self.torch.empty(workspace_size(n), dtype=self.torch.uint8, device="cuda")
            self._ws[n] = ws
        return ws

    def solve(self, D, E, W, diagnostics: bool = False):
        n = D.shape[0]
        ws = self.workspace(n)
        st = _load().ref_solve(
            self.h, n, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(E.data_ptr()),
            ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
            1 if diagnostics else 0,
        )
        if st != 0:
            raise RuntimeError(f"reference solve status {st}")
        return W

    def level_diagnostics(self):
        out = np.zeros(8 * 40, dtype=np.int32)
        k = _load().ref_level_diagnostics(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 40)
        names = ("merge_count", "size_sum", "dd_before_sum", "dd_after_sum", "dd_after_max",
                 "secular_iter_sum", "secular_iter_max", "secular_iter_failed")
        return [dict(zip(names, (int(v) for v in out[8 * i:8 * i + 8]))) for i in range(k)]
