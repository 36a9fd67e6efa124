"""brdc -- host-side mirror of the reference's tridiagonal-solver interface.

Python bindings (ctypes) for ``libbrdc_b200.so``, the sm_100a boundary-row
(BR) values-only divide-and-conquer eigensolver.  The functions mirror the
reference's entry points:

* :func:`workspace_size` -- ``tridiag_solver_workspace_size``
  (gpu/src/tridiag_solver.cu:2373)
* :meth:`Solver.dstebr` -- ``tridiag_solver_run_from_device_tridiagonal``
  (gpu/src/tridiag_solver.cu:2541): device D, E in, ascending W out
* :func:`dstedc_dc_br` -- ``DSTEDC_DC_BR`` (cpu/src/dstedc_dc_br.f:7), the
  LAPACK-style host entry with the LWORK/LIWORK = -1 query

Device memory and streams come from PyTorch; the library itself takes raw
pointers only.  There is no CPU fallback: every function raises when the
compiled library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbrdc_b200.so")

STATUS = {
    0: "success",
    1: "invalid_handle",
    2: "invalid_pointer",
    3: "invalid_value",
    4: "invalid_workspace",
    5: "alloc_failed",
    6: "cuda_error",
    7: "internal_error",
    8: "not_implemented",
    9: "not_converged",
}
SUCCESS, INVALID_HANDLE, INVALID_POINTER, INVALID_VALUE, INVALID_WORKSPACE = 0, 1, 2, 3, 4
ALLOC_FAILED, CUDA_ERROR, INTERNAL_ERROR, NOT_IMPLEMENTED, NOT_CONVERGED = 5, 6, 7, 8, 9
FLAG_KEEP_CHECKPOINTS = 1
MAX_LEVELS = 40

# Every entry point declared in include/brdc.h.
EXPORTS = (
    "brdc_create",
    "brdc_destroy",
    "brdc_set_stream",
    "brdc_get_stream",
    "brdc_get_last_error",
    "brdc_status_to_string",
    "brdc_dstebr_workspace_size",
    "brdc_dstebr",
    "brdc_dstebr_backward",
    "brdc_get_info",
    "brdc_get_diagnostics",
    "brdc_dstedc_dc_br_",
    "brdc_dstebr_batched_workspace_size",
    "brdc_dstebr_batched",
    "brdc_version",
    "brdc_set_timing",
    "brdc_get_last_timings",
    "brdc_dstebr_noalloc",
    "brdc_dstebr_batched_checkpoint_workspace_size",
    "brdc_dstebr_batched_backward",
    "brdc_set_tuning",
    "brdc_get_tuning",
    "brdc_autotune",
    "brdc_dstebr_vectors_workspace_size",
    "brdc_dstebr_vectors",
    "brdc_set_limits",
    "brdc_get_limits",
    "brdc_dstebr_noalloc_get_info",
    "brdc_get_merge_trace",
    "brdc_set_graphs",
    "brdc_get_last_launches",
    "brdc_dstebr_host_workspace_size",
    "brdc_dstebr_host",
)


class BrdcError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {STATUS.get(status, status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class LevelDiag(ctypes.Structure):
    _fields_ = [
        (name, ctypes.c_int)
        for name in (
            "level", "merge_count", "size_sum", "dd_before_sum", "dd_after_sum",
            "dd_after_max", "zero_deflated_total", "close_deflated_total",
            "secular_iter_sum", "secular_iter_max", "secular_iter_failed",
            "threads_per_root",
        )
    ] + [("dd_after_sq_sum", ctypes.c_longlong)]


class Diagnostics(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int),
        ("levels", ctypes.c_int),
        ("leaf_count", ctypes.c_int),
        ("leaf_sweeps_max", ctypes.c_int),
        ("leaf_sweeps_sum", ctypes.c_int),
        ("level", LevelDiag * MAX_LEVELS),
    ]

    def as_dict(self) -> dict:
        out = {
            "n": self.n,
            "levels": self.levels,
            "leaf_count": self.leaf_count,
            "leaf_sweeps_max": self.leaf_sweeps_max,
            "leaf_sweeps_sum": self.leaf_sweeps_sum,
            "level": [],
        }
        for k in range(self.levels):
            lv = self.level[k]
            out["level"].append({f: getattr(lv, f) for f, _ in LevelDiag._fields_})
        return out


class Tuning(ctypes.Structure):
    _fields_ = [
        ("subtree_levels", ctypes.c_int),
        ("deflate_cluster", ctypes.c_int),
        ("sweep_lanes_target", ctypes.c_int),
        ("fused_level_rows", ctypes.c_int),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Limits(ctypes.Structure):
    _fields_ = [
        ("secular_max_iter", ctypes.c_int),
        ("reserved", ctypes.c_int),
        ("wait_limit_ns", ctypes.c_longlong),
    ]

    def as_dict(self) -> dict:
        return {"secular_max_iter": self.secular_max_iter, "wait_limit_ns": self.wait_limit_ns}


class Timings(ctypes.Structure):
    _fields_ = [
        ("total_ms", ctypes.c_float),
        ("init_ms", ctypes.c_float),
        ("leaf_ms", ctypes.c_float),
        ("merge_ms", ctypes.c_float),
        ("secular_ms", ctypes.c_float),
        ("lowner_ms", ctypes.c_float),
        ("rows_ms", ctypes.c_float),
        ("launches", ctypes.c_int),
        ("levels", ctypes.c_int),
        ("level_ms", (ctypes.c_float * 4) * MAX_LEVELS),
        ("fused_levels", ctypes.c_int),
    ]

    def as_dict(self) -> dict:
        out = {f: getattr(self, f) for f, _ in self._fields_ if f != "level_ms"}
        out["level_ms"] = [list(self.level_ms[k]) for k in range(self.levels)]
        return out


_lib = None


def load() -> ctypes.CDLL:
    """Load the compiled library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with build.py (there is no fallback)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    vp, sz, i64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int64
    ip = ctypes.POINTER(ctypes.c_int)
    lib.brdc_create.argtypes = [ctypes.POINTER(vp)]
    lib.brdc_destroy.argtypes = [vp]
    lib.brdc_set_stream.argtypes = [vp, vp]
    lib.brdc_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.brdc_get_last_error.argtypes = [vp, ip, ip, ctypes.POINTER(ctypes.c_char_p)]
    lib.brdc_status_to_string.argtypes = [ctypes.c_int]
    lib.brdc_status_to_string.restype = ctypes.c_char_p
    lib.brdc_dstebr_workspace_size.argtypes = [i64, ctypes.c_int, ctypes.POINTER(sz)]
    lib.brdc_dstebr.argtypes = [vp, i64, vp, vp, vp, vp, sz]
    lib.brdc_dstebr_backward.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, sz, ctypes.c_int]
    lib.brdc_get_info.argtypes = [vp, vp, ip]
    lib.brdc_get_diagnostics.argtypes = [vp, vp, ctypes.POINTER(Diagnostics)]
    lib.brdc_dstedc_dc_br_.argtypes = [
        ip, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
        ctypes.POINTER(ctypes.c_double), ip, ip, ip, ip,
    ]
    lib.brdc_dstedc_dc_br_.restype = None
    lib.brdc_dstebr_batched_workspace_size.argtypes = [i64, ctypes.POINTER(i64), ctypes.POINTER(sz)]
    lib.brdc_dstebr_batched.argtypes = [vp, i64, ctypes.POINTER(i64), vp, vp, vp, vp, sz]
    lib.brdc_dstebr_batched_checkpoint_workspace_size.argtypes = [
        i64, ctypes.POINTER(i64), ctypes.POINTER(sz)]
    lib.brdc_dstebr_batched_backward.argtypes = [
        vp, i64, ctypes.POINTER(i64), vp, vp, vp, vp, vp, vp, sz, ctypes.c_int]
    lib.brdc_version.restype = ctypes.c_char_p
    lib.brdc_set_timing.argtypes = [vp, ctypes.c_int]
    lib.brdc_dstebr_noalloc.argtypes = [vp, i64, vp, vp, vp]
    lib.brdc_dstebr_vectors_workspace_size.argtypes = [i64, ctypes.POINTER(sz)]
    lib.brdc_dstebr_vectors.argtypes = [vp, i64, vp, vp, vp, vp, i64, vp, sz]
    lib.brdc_get_last_timings.argtypes = [vp, ctypes.POINTER(Timings)]
    lib.brdc_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    lib.brdc_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    lib.brdc_autotune.argtypes = [vp, i64, ctypes.POINTER(i64), vp, vp, vp, vp, sz,
                                  ctypes.POINTER(Tuning)]
    lib.brdc_set_limits.argtypes = [vp, ctypes.POINTER(Limits)]
    lib.brdc_dstebr_noalloc_get_info.argtypes = [vp, ip]
    dpp = ctypes.POINTER(ctypes.c_double)
    lib.brdc_get_merge_trace.argtypes = [vp, vp, sz, i64, ctypes.c_int, dpp, dpp, ip, ip, ip,
                                         dpp, dpp, ip, dpp, dpp]
    lib.brdc_get_limits.argtypes = [vp, ctypes.POINTER(Limits)]
    lib.brdc_set_graphs.argtypes = [vp, ctypes.c_int]
    lib.brdc_get_last_launches.argtypes = [vp, ip, ip]
    lib.brdc_dstebr_host_workspace_size.argtypes = [i64, ctypes.POINTER(sz)]
    lib.brdc_dstebr_host.argtypes = [vp, i64, vp, vp, vp, vp, sz]
    for f in ("brdc_create", "brdc_destroy", "brdc_set_stream", "brdc_get_stream",
              "brdc_get_last_error", "brdc_dstebr_workspace_size", "brdc_dstebr",
              "brdc_dstebr_backward", "brdc_get_info", "brdc_get_diagnostics",
              "brdc_dstebr_batched_workspace_size", "brdc_dstebr_batched",
              "brdc_set_timing", "brdc_get_last_timings", "brdc_dstebr_noalloc",
              "brdc_dstebr_batched_checkpoint_workspace_size", "brdc_dstebr_batched_backward",
              "brdc_set_tuning", "brdc_get_tuning", "brdc_autotune",
              "brdc_set_limits", "brdc_get_limits", "brdc_dstebr_noalloc_get_info",
              "brdc_get_merge_trace", "brdc_set_graphs", "brdc_get_last_launches",
              "brdc_dstebr_host_workspace_size", "brdc_dstebr_host"):
        getattr(lib, f).restype = ctypes.c_int
    _lib = lib
    return lib


def _check(status: int, where: str, handle=None) -> None:
    if status != SUCCESS:
        detail = ""
        if handle is not None:
            code = ctypes.c_int()
            src = ctypes.c_int()
            site = ctypes.c_char_p()
            load().brdc_get_last_error(handle, ctypes.byref(code), ctypes.byref(src), ctypes.byref(site))
            if site.value:
                detail = f"code={code.value} site={site.value.decode()}"
        raise BrdcError(status, where, detail)


def workspace_size(n: int, flags: int = 0) -> int:
    """Bytes of device workspace for one solve of order n."""
    out = ctypes.c_size_t()
    _check(load().brdc_dstebr_workspace_size(int(n), int(flags), ctypes.byref(out)), "workspace_size")
    return int(out.value)


def batched_workspace_size(offsets: Sequence[int], checkpoints: bool = False) -> int:
    """Bytes of device workspace for one batched solve; with checkpoints,
    the size that also records what the batched backward reads."""
    off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64))
    out = ctypes.c_size_t()
    fn = (load().brdc_dstebr_batched_checkpoint_workspace_size if checkpoints
          else load().brdc_dstebr_batched_workspace_size)
    _check(fn(len(off) - 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(out)),
           "batched_workspace_size")
    return int(out.value)


class Solver:
    """One handle plus cached workspaces; runs on the current torch stream
    unless ``stream`` is given."""

    def __init__(self, stream=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("brdc needs a CUDA device")
        self._torch = torch
        lib = load()
        h = ctypes.c_void_p()
        _check(lib.brdc_create(ctypes.byref(h)), "brdc_create")
        self.h = h
        self._ws = {}
        self.set_stream(stream)

    def close(self) -> None:
        if getattr(self, "h", None):
            load().brdc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream=None) -> None:
        torch = self._torch
        s = stream if stream is not None else torch.cuda.current_stream()
        self.stream = s
        _check(load().brdc_set_stream(self.h, ctypes.c_void_p(s.cuda_stream)), "set_stream", self.h)

    def tuning(self) -> dict:
        t = Tuning()
        _check(load().brdc_get_tuning(self.h, ctypes.byref(t)), "get_tuning", self.h)
        return t.as_dict()

    def set_tuning(self, **kw) -> None:
        """Change launch-shape parameters (subtree_levels, deflate_cluster,
        sweep_lanes_target, fused_level_rows); the others keep their values."""
        cur = self.tuning()
        cur.update(kw)
        t = Tuning(**cur)
        _check(load().brdc_set_tuning(self.h, ctypes.byref(t)), "set_tuning", self.h)

    def limits(self) -> dict:
        lim = Limits()
        _check(load().brdc_get_limits(self.h, ctypes.byref(lim)), "get_limits", self.h)
        return lim.as_dict()

    def set_limits(self, **kw) -> None:
        """Change failure limits (secular_max_iter, wait_limit_ns); the
        others keep their values."""
        cur = self.limits()
        cur.update(kw)
        lim = Limits(secular_max_iter=int(cur["secular_max_iter"]), reserved=0,
                     wait_limit_ns=int(cur["wait_limit_ns"]))
        _check(load().brdc_set_limits(self.h, ctypes.byref(lim)), "set_limits", self.h)

    def last_error(self):
        """(code, source, site) of the handle's last recorded error."""
        code, src, site = ctypes.c_int(), ctypes.c_int(), ctypes.c_char_p()
        load().brdc_get_last_error(self.h, ctypes.byref(code), ctypes.byref(src), ctypes.byref(site))
        return code.value, src.value, (site.value.decode() if site.value else None)

    def autotune(self, D, E, offsets=None, workspace=None) -> dict:
        """Time this input (one matrix, or a packed batch with offsets) under
        candidate launch shapes and keep the fastest on the handle."""
        torch = self._torch
        n = D.shape[0]
        off = np.ascontiguousarray(np.asarray([0, n] if offsets is None else offsets,
                                              dtype=np.int64))
        if offsets is None:
            ws = self.workspace(n) if workspace is None else workspace
            Ep = E.contiguous() if E is not None and E.numel() > 0 else D
        else:
            ws = self.batched_workspace(off) if workspace is None else workspace
            Ep = E.contiguous()
        W = torch.empty(int(off[-1]), dtype=torch.float64, device=D.device)
        t = Tuning()
        st = load().brdc_autotune(
            self.h, len(off) - 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            ctypes.c_void_p(D.contiguous().data_ptr()), ctypes.c_void_p(Ep.data_ptr()),
            ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
            ctypes.byref(t))
        _check(st, "brdc_autotune", self.h)
        return t.as_dict()

    def set_timing(self, enable: bool) -> None:
        _check(load().brdc_set_timing(self.h, 1 if enable else 0), "set_timing", self.h)

    def last_timings(self) -> dict:
        t = Timings()
        _check(load().brdc_get_last_timings(self.h, ctypes.byref(t)), "get_last_timings", self.h)
        return t.as_dict()

    def set_graphs(self, enable: bool) -> None:
        """Graph replay of repeated plain solves (brdc_set_graphs; on by
        default)."""
        _check(load().brdc_set_graphs(self.h, 1 if enable else 0), "set_graphs", self.h)

    def last_launches(self) -> dict:
        """Kernels the last plain solve ran, and whether it was a graph
        replay (brdc_get_last_launches; synchronises the stream)."""
        n = ctypes.c_int(0)
        r = ctypes.c_int(0)
        _check(load().brdc_get_last_launches(self.h, ctypes.byref(n), ctypes.byref(r)),
               "get_last_launches", self.h)
        return {"launches": n.value, "replayed": bool(r.value)}

    def workspace(self, n: int, flags: int = 0):
        key = ("single", int(n), int(flags))
        ws = self._ws.get(key)
        if ws is None:
            nbytes = workspace_size(n, flags)
            ws = self._torch.empty(nbytes, dtype=self._torch.uint8, device="cuda")
            self._ws[key] = ws
        return ws

    def dstebr(self, D, E, W=None, workspace=None):
        """Eigenvalues (ascending, float64, on the device) of the symmetric
        tridiagonal with diagonal D[n] and off-diagonal E[n-1]."""
        torch = self._torch
        n = D.shape[0]
        if D.dtype != torch.float64 or not D.is_cuda:
            raise TypeError("D must be a float64 CUDA tensor")
        D = D.contiguous()
        E = E.contiguous() if E is not None and E.numel() > 0 else D  # unused for n == 1
        if W is None:
            W = torch.empty(n, dtype=torch.float64, device=D.device)
        ws = self.workspace(n) if workspace is None else workspace
        st = load().brdc_dstebr(
            self.h, n, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(E.data_ptr()),
            ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
        )
        _check(st, "brdc_dstebr", self.h)
        return W

    def host_workspace(self, n: int):
        """Device workspace of dstebr_host (brdc_dstebr_host_workspace_size)."""
        key = ("host", int(n))
        ws = self._ws.get(key)
        if ws is None:
            nb = ctypes.c_size_t(0)
            _check(load().brdc_dstebr_host_workspace_size(int(n), ctypes.byref(nb)),
                   "brdc_dstebr_host_workspace_size")
            ws = self._torch.empty(nb.value, dtype=self._torch.uint8, device="cuda")
            self._ws[key] = ws
        return ws

    def dstebr_host(self, D, E, W=None, workspace=None):
        """dstebr on host (CPU) float64 tensors: D and E are copied in, the
        eigenvalues copied back into W (allocated pinned when None).  The call
        only enqueues; W is valid once the handle's stream has synchronised.
        Pinned tensors (pin_memory()) keep it from blocking the host
        (brdc_dstebr_host)."""
        torch = self._torch
        n = D.shape[0]
        if D.dtype != torch.float64 or D.is_cuda or not D.is_contiguous():
            raise TypeError("D must be a contiguous float64 CPU tensor")
        if n > 1 and (E is None or E.dtype != torch.float64 or E.is_cuda or not E.is_contiguous()):
            raise TypeError("E must be a contiguous float64 CPU tensor")
        if W is None:
            W = torch.empty(n, dtype=torch.float64).pin_memory()
        ws = self.host_workspace(n) if workspace is None else workspace
        e_ptr = E.data_ptr() if n > 1 else None
        st = load().brdc_dstebr_host(self.h, n, ctypes.c_void_p(D.data_ptr()),
                                     ctypes.c_void_p(e_ptr), ctypes.c_void_p(W.data_ptr()),
                                     ctypes.c_void_p(ws.data_ptr()), ws.numel())
        _check(st, "brdc_dstebr_host", self.h)
        return W

    def dstebr_vectors(self, D, E, workspace=None):
        """Eigenvalues W[n] (ascending) and eigenvectors Z (n x n, column j
        for W[j]) on the device (brdc_dstebr_vectors)."""
        torch = self._torch
        n = D.shape[0]
        if D.dtype != torch.float64 or not D.is_cuda:
            raise TypeError("D must be a float64 CUDA tensor")
        D = D.contiguous()
        E = E.contiguous() if E is not None and E.numel() > 0 else D
        W = torch.empty(n, dtype=torch.float64, device=D.device)
        Zt = torch.empty((n, n), dtype=torch.float64, device=D.device)  # row-major Z^T
        if workspace is None:
            nb = ctypes.c_size_t(0)
            _check(load().brdc_dstebr_vectors_workspace_size(n, ctypes.byref(nb)),
                   "brdc_dstebr_vectors_workspace_size")
            workspace = torch.empty(nb.value, dtype=torch.uint8, device=D.device)
        st = load().brdc_dstebr_vectors(
            self.h, n, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(E.data_ptr()),
            ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(Zt.data_ptr()), n,
            ctypes.c_void_p(workspace.data_ptr()), workspace.numel(),
        )
        _check(st, "brdc_dstebr_vectors", self.h)
        return W, Zt.t()

    def checkpoint_workspace(self, n: int):
        """Workspace that also records the per-level state the adjoint reads
        (cached per order on this solver: the next solve of order n on it
        overwrites the checkpoints)."""
        return self.workspace(n, FLAG_KEEP_CHECKPOINTS)

    def new_checkpoint_workspace(self, n: int):
        """A fresh, uncached checkpointing workspace for one solve of order n."""
        nbytes = workspace_size(n, FLAG_KEEP_CHECKPOINTS)
        return self._torch.empty(nbytes, dtype=self._torch.uint8, device="cuda")

    def dstebr_backward(self, D, E, G, workspace=None, keep_forward: bool = False,
                        gD=None, gE=None):
        """dL/dD, dL/dE for L = sum(G * W).  With keep_forward the workspace
        must hold the checkpoints of a brdc_dstebr call on the same D, E;
        otherwise the forward solve is re-run first."""
        torch = self._torch
        n = D.shape[0]
        D = D.contiguous()
        E = E.contiguous() if E is not None and E.numel() > 0 else D
        G = G.contiguous()
        if gD is None:
            gD = torch.empty(n, dtype=torch.float64, device=D.device)
        if gE is None:
            gE = torch.empty(max(n - 1, 1), dtype=torch.float64, device=D.device)
        ws = self.checkpoint_workspace(n) if workspace is None else workspace
        st = load().brdc_dstebr_backward(
            self.h, n, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(E.data_ptr()),
            ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(gD.data_ptr()),
            ctypes.c_void_p(gE.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
            1 if keep_forward else 0,
        )
        _check(st, "brdc_dstebr_backward", self.h)
        return gD, gE[: max(n - 1, 0)]

    def dstebr_noalloc(self, D, E, W=None):
        """Solve with the library's static scratch (n <= 16384); no
        workspace is allocated by anyone."""
        torch = self._torch
        n = D.shape[0]
        D = D.contiguous()
        E = E.contiguous() if E is not None and E.numel() > 0 else D
        if W is None:
            W = torch.empty(n, dtype=torch.float64, device=D.device)
        st = load().brdc_dstebr_noalloc(self.h, n, ctypes.c_void_p(D.data_ptr()),
                                        ctypes.c_void_p(E.data_ptr()), ctypes.c_void_p(W.data_ptr()))
        _check(st, "brdc_dstebr_noalloc", self.h)
        return W

    def noalloc_info_status(self):
        """(info, status) of the last allocation-free solve on this device."""
        out = ctypes.c_int()
        st = load().brdc_dstebr_noalloc_get_info(self.h, ctypes.byref(out))
        if st not in (SUCCESS, NOT_CONVERGED, INTERNAL_ERROR):
            _check(st, "brdc_dstebr_noalloc_get_info", self.h)
        return int(out.value), int(st)

    def info(self, n: int, workspace=None) -> int:
        """Device status of the last solve on the workspace: 0, the number of
        unconverged roots (> 0), or a negative device error code."""
        return self.info_status(n, workspace)[0]

    def info_status(self, n: int, workspace=None):
        """(info, status) of brdc_get_info for the workspace."""
        ws = self.workspace(n) if workspace is None else workspace
        out = ctypes.c_int()
        st = load().brdc_get_info(self.h, ctypes.c_void_p(ws.data_ptr()), ctypes.byref(out))
        if st not in (SUCCESS, NOT_CONVERGED, INTERNAL_ERROR):
            _check(st, "brdc_get_info", self.h)
        return int(out.value), int(st)

    def merge_trace(self, n: int, level: int, workspace) -> dict:
        """Deflation record of one merge level of the last solve on a
        checkpointing workspace (brdc_get_merge_trace), as numpy arrays."""
        L = self.diagnostics(n, workspace)["levels"]
        nodes = 1 << (L - 1 - level)
        out = {k: np.zeros(n) for k in ("d", "z", "c", "s")}
        out.update({k: np.zeros(n, dtype=np.int32) for k in ("row", "state", "link")})
        out["K"] = np.zeros(nodes, dtype=np.int32)
        out["rho"] = np.zeros(nodes)
        out["tol"] = np.zeros(nodes)
        dp = ctypes.POINTER(ctypes.c_double)
        ipt = ctypes.POINTER(ctypes.c_int)
        st = load().brdc_get_merge_trace(
            self.h, ctypes.c_void_p(workspace.data_ptr()), workspace.numel(), int(n), int(level),
            out["d"].ctypes.data_as(dp), out["z"].ctypes.data_as(dp), out["row"].ctypes.data_as(ipt),
            out["state"].ctypes.data_as(ipt), out["link"].ctypes.data_as(ipt),
            out["c"].ctypes.data_as(dp), out["s"].ctypes.data_as(dp), out["K"].ctypes.data_as(ipt),
            out["rho"].ctypes.data_as(dp), out["tol"].ctypes.data_as(dp))
        _check(st, "brdc_get_merge_trace", self.h)
        return out

    def diagnostics(self, n: int, workspace=None) -> dict:
        ws = self.workspace(n) if workspace is None else workspace
        d = Diagnostics()
        _check(load().brdc_get_diagnostics(self.h, ctypes.c_void_p(ws.data_ptr()), ctypes.byref(d)),
               "brdc_get_diagnostics", self.h)
        return d.as_dict()

    # ------------------------------------------------------------ batched
    def batched_workspace(self, offsets, checkpoints: bool = False):
        off = tuple(int(x) for x in offsets)
        key = ("batched", checkpoints, off)
        ws = self._ws.get(key)
        if ws is None:
            nbytes = batched_workspace_size(off, checkpoints)
            ws = self._torch.empty(nbytes, dtype=self._torch.uint8, device="cuda")
            self._ws[key] = ws
        return ws

    def dstebr_batched(self, offsets, D, E, W=None, workspace=None):
        """Solve every tridiagonal packed in D/E (instance b occupies rows
        offsets[b]:offsets[b+1]); returns W packed the same way."""
        torch = self._torch
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64))
        total = int(off[-1])
        if W is None:
            W = torch.empty(total, dtype=torch.float64, device=D.device)
        ws = self.batched_workspace(off) if workspace is None else workspace
        st = load().brdc_dstebr_batched(
            self.h, len(off) - 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(E.data_ptr()),
            ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
        )
        _check(st, "brdc_dstebr_batched", self.h)
        return W

    def dstebr_batched_backward(self, offsets, D, E, G, workspace=None,
                                keep_forward: bool = False, gD=None, gE=None):
        """dL/dD, dL/dE of L = sum(G * W) for a packed batch (layout of
        dstebr_batched).  keep_forward reuses the checkpoints that a
        dstebr_batched call with the same checkpoint workspace recorded."""
        torch = self._torch
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64))
        total = int(off[-1])
        if gD is None:
            gD = torch.empty(total, dtype=torch.float64, device=D.device)
        if gE is None:
            gE = torch.empty(total, dtype=torch.float64, device=D.device)
        ws = self.batched_workspace(off, True) if workspace is None else workspace
        st = load().brdc_dstebr_batched_backward(
            self.h, len(off) - 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(E.data_ptr()),
            ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(gD.data_ptr()),
            ctypes.c_void_p(gE.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
            1 if keep_forward else 0,
        )
        _check(st, "brdc_dstebr_batched_backward", self.h)
        return gD, gE


def dstedc_dc_br(d, e) -> np.ndarray:
    """LAPACK-style host call (DSTEDC_DC_BR argument list): host d, e in,
    ascending eigenvalues out; the work runs on the GPU."""
    lib = load()
    d = np.array(d, dtype=np.float64, copy=True)
    n = d.shape[0]
    e = np.concatenate([np.array(e, dtype=np.float64)[: max(n - 1, 0)], np.zeros(1)])
    nn = ctypes.c_int(n)
    wq = np.zeros(1)
    iwq = np.zeros(1, dtype=np.int32)
    m1 = ctypes.c_int(-1)
    info = ctypes.c_int(0)
    dp = ctypes.POINTER(ctypes.c_double)
    ipt = ctypes.POINTER(ctypes.c_int)
    lib.brdc_dstedc_dc_br_(ctypes.byref(nn), d.ctypes.data_as(dp), e.ctypes.data_as(dp),
                           wq.ctypes.data_as(dp), ctypes.byref(m1), iwq.ctypes.data_as(ipt),
                           ctypes.byref(m1), ctypes.byref(info))
    if info.value != 0:
        raise BrdcError(INVALID_VALUE, "dstedc_dc_br query", f"INFO={info.value}")
    lw, liw = max(1, int(wq[0])), max(1, int(iwq[0]))
    work = np.zeros(lw)
    iwork = np.zeros(liw, dtype=np.int32)
    lwc, liwc = ctypes.c_int(lw), ctypes.c_int(liw)
    lib.brdc_dstedc_dc_br_(ctypes.byref(nn), d.ctypes.data_as(dp), e.ctypes.data_as(dp),
                           work.ctypes.data_as(dp), ctypes.byref(lwc), iwork.ctypes.data_as(ipt),
                           ctypes.byref(liwc), ctypes.byref(info))
    if info.value != 0:
        raise BrdcError(NOT_CONVERGED if info.value > 0 else INVALID_VALUE,
                        "dstedc_dc_br", f"INFO={info.value}")
    return d


def dstedc_dc_br_query(n: int, lwork: int = -1, liwork: int = -1):
    """Raw LAPACK-style call for the argument checks: returns
    (INFO, WORK(1), IWORK(1)) without solving (queries or bad arguments)."""
    lib = load()
    nn = ctypes.c_int(int(n))
    w = np.zeros(max(1, 1))
    iw = np.zeros(1, dtype=np.int32)
    lwc, liwc, info = ctypes.c_int(lwork), ctypes.c_int(liwork), ctypes.c_int(0)
    dp = ctypes.POINTER(ctypes.c_double)
    d = np.zeros(max(int(n), 1))
    e = np.zeros(max(int(n), 1))
    lib.brdc_dstedc_dc_br_(ctypes.byref(nn), d.ctypes.data_as(dp), e.ctypes.data_as(dp),
                           w.ctypes.data_as(dp), ctypes.byref(lwc),
                           iw.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(liwc),
                           ctypes.byref(info))
    return int(info.value), int(w[0]), int(iw[0])


_default_solver: Optional[Solver] = None


def dstebr(D, E):
    """Module-level convenience: eigenvalues of (D, E) on the current stream."""
    global _default_solver
    if _default_solver is None:
        _default_solver = Solver()
    else:
        _default_solver.set_stream()
    return _default_solver.dstebr(D, E)
