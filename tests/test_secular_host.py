"""The product's per-root secular state machine, compiled for the host,
against LAPACK DLAED4 (the routine the reference calls per root,
cpu/src/dlaed4_br.f:59)."""
import ctypes
import zlib

import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module")
def hostlib(built_lib):
    import build as b

    lib = ctypes.CDLL(b.HOSTLIB)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.brdc_host_secular_root.argtypes = [
        ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
        ctypes.POINTER(ctypes.c_int), dp, ctypes.POINTER(ctypes.c_int),
    ]
    return lib


def _root(lib, d, z, rho, i):
    dp = ctypes.POINTER(ctypes.c_double)
    org, tau, f = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
    sweeps = lib.brdc_host_secular_root(len(d), d.ctypes.data_as(dp), z.ctypes.data_as(dp),
                                        rho, float(z @ z), i, ctypes.byref(org),
                                        ctypes.byref(tau), ctypes.byref(f))
    return d[org.value] + tau.value, sweeps, f.value


@pytest.mark.parametrize("kind", ["normal", "uniform", "clustered", "tiny_z"])
def test_roots_match_dlaed4(hostlib, kind):
    rng = np.random.default_rng(zlib.crc32(kind.encode()))
    worst, sw_max = 0.0, 0
    for _ in range(40):
        K = int(rng.integers(2, 200))
        if kind == "normal":
            d = np.sort(rng.standard_normal(K))
        elif kind == "uniform":
            d = np.sort(rng.uniform(0, 1, K))
        elif kind == "clustered":
            d = np.unique(np.concatenate([rng.uniform(-1, 1, K // 2), 0.3 + 1e-8 * rng.uniform(-1, 1, K - K // 2)]))
            K = d.shape[0]
        else:
            d = np.sort(rng.standard_normal(K))
        z = rng.standard_normal(K)
        if kind == "tiny_z":
            z[::2] *= 1e-7
        z /= np.linalg.norm(z)
        rho = float(rng.uniform(0.05, 4.0))
        for i in range(K):
            lam_ref, _ = oracle.dlaed4(d, z, rho, i)
            lam, sweeps, failed = _root(hostlib, d, z, rho, i)
            assert not failed
            # accurate relative to the distance to the nearest pole, or
            # normwise (relative to max(|lambda|, max|d|)): a root near zero
            # has no relative accuracy in |lambda| (nor has DLAED4's), and
            # with many tiny weights the secular function's own rounding
            # can exceed 1e-12 of the gap
            gap = float(np.min(np.abs(d - lam_ref)))
            diff = abs(lam - lam_ref)
            rel_gap = diff / gap if gap > 0 else np.inf
            rel_norm = diff / max(abs(lam_ref), float(np.max(np.abs(d))))
            worst = max(worst, min(rel_gap, rel_norm))
            sw_max = max(sw_max, sweeps)
            if i < K - 1:
                assert d[i] <= lam <= d[i + 1]
            else:
                assert lam >= d[K - 1]
    assert worst < 1e-12
    assert sw_max <= 20


def test_two_poles_closed_form(hostlib):
    d = np.array([0.0, 1.0])
    z = np.array([0.6, 0.8])
    rho = 1.5
    M = np.diag(d) + rho * np.outer(z, z)
    ev = np.linalg.eigvalsh(M)
    for i in range(2):
        lam, _, _ = _root(hostlib, d, z, rho, i)
        assert abs(lam - ev[i]) < 1e-15 * 4


def _root_capped(lib, d, z, rho, i, max_iter):
    dp = ctypes.POINTER(ctypes.c_double)
    lib.brdc_host_secular_root_capped.argtypes = [
        ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
        ctypes.POINTER(ctypes.c_int), dp, ctypes.POINTER(ctypes.c_int),
    ]
    org, tau, f = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
    sweeps = lib.brdc_host_secular_root_capped(len(d), d.ctypes.data_as(dp), z.ctypes.data_as(dp),
                                               rho, float(np.nansum(z * z)), i, max_iter,
                                               ctypes.byref(org), ctypes.byref(tau), ctypes.byref(f))
    return sweeps, f.value


def test_iteration_cap_reports_failure(hostlib):
    """With a cap of one iteration no root of a generic problem converges:
    every one stops and is flagged; with the default cap none is."""
    rng = np.random.default_rng(21)
    K = 60
    d = np.sort(rng.standard_normal(K))
    z = rng.standard_normal(K)
    z /= np.linalg.norm(z)
    flagged = 0
    for i in range(K):
        sweeps, failed = _root_capped(hostlib, d, z, 1.0, i, 1)
        assert sweeps <= 2
        flagged += failed
        assert _root_capped(hostlib, d, z, 1.0, i, 64)[1] == 0
    assert flagged == K


def test_nan_secular_function_is_a_failure(hostlib):
    """A NaN in the data makes the secular function NaN: the root must stop
    and be reported failed, not accepted as converged."""
    d = np.array([0.0, 0.5, 1.0, 2.0])
    z = np.array([0.5, np.nan, 0.5, 0.5])
    for i in range(len(d)):
        sweeps, failed = _root_capped(hostlib, d, z, 1.0, i, 64)
        assert failed == 1
        assert sweeps <= 2
