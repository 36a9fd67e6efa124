"""Failure statuses of the device solve, reached on purpose without
faulting the GPU.

* An iteration cap of one makes secular roots stop unconverged:
  brdc_get_info returns NOT_CONVERGED with info > 0 (the reference only
  counts such roots in its diagnostics, gpu/src/tridiag_solver.cu:2351-2370).
* A wait limit of zero makes the bounded waits of the per-level sweep kernel
  (grid barriers, tile-copy mbarriers) give up at once: the kernel records
  the timeout in the workspace status word, waits for its own copies in
  flight, and every later kernel returns at once; brdc_get_info returns
  INTERNAL_ERROR with info < 0, and the same handle then solves normally.
* A NaN or an infinity in D or E is caught before anything is solved
  (info = -4), for a single solve and for a batch.
Every wait these tests exhaust is one the kernels bound themselves; none
relies on a trap, a fault or a hang.
"""
import numpy as np
import pytest

import brdc
import oracle
from brdc import families

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture()
def fresh():
    s = brdc.Solver()
    yield s
    s.close()


def solve(s, d, e, ws=None):
    import torch

    W = s.dstebr(torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda"), workspace=ws)
    return W


def test_default_limits(fresh):
    assert fresh.limits() == {"secular_max_iter": 64, "wait_limit_ns": 20_000_000_000}


def test_limits_reject_out_of_range(fresh):
    for kw in ({"secular_max_iter": 0}, {"secular_max_iter": 1001}, {"wait_limit_ns": -1},
               {"wait_limit_ns": 10**12 + 1}):
        with pytest.raises(brdc.BrdcError) as ex:
            fresh.set_limits(**kw)
        assert ex.value.status == brdc.INVALID_VALUE
    assert fresh.limits()["secular_max_iter"] == 64


def test_iteration_cap_reports_not_converged(fresh):
    n = 4096
    d, e = families.generate("normal", n)
    fresh.set_limits(secular_max_iter=1)
    solve(fresh, d, e)
    info, st = fresh.info_status(n)
    assert st == brdc.NOT_CONVERGED
    assert info > 0
    diag = fresh.diagnostics(n)
    assert sum(lv["secular_iter_failed"] for lv in diag["level"]) == info
    # the default cap again: converged and correct
    fresh.set_limits(secular_max_iter=64)
    W = solve(fresh, d, e).cpu().numpy()
    assert fresh.info_status(n) == (0, brdc.SUCCESS)
    ref = oracle.dstedc_dc_br(d, e)
    assert np.max(np.abs(W - ref)) < TOL * np.max(np.abs(ref))


@pytest.mark.parametrize("n", [16384])
def test_wait_limit_stops_the_solve_and_the_handle_recovers(fresh, n):
    """Toeplitz of order 16384 keeps 8192 poles at the top merge, so its
    last levels run in the sweep kernel: tile copies (CTA role) and grid
    barriers.  With a zero wait limit those waits give up."""
    d, e = families.generate("toeplitz", n)
    fresh.set_limits(wait_limit_ns=0)
    solve(fresh, d, e)
    info, st = fresh.info_status(n)
    assert st == brdc.INTERNAL_ERROR
    assert info in (-1, -3)
    code, src, site = fresh.last_error()
    assert src == 2 and code == -info  # BRDC_ERROR_SRC_DEVICE
    # the context is intact: the default limit solves the same input
    fresh.set_limits(wait_limit_ns=20_000_000_000)
    W = solve(fresh, d, e).cpu().numpy()
    assert fresh.info_status(n) == (0, brdc.SUCCESS)
    ref = families.toeplitz_eigenvalues(n)
    assert np.max(np.abs(W - ref)) < TOL * 4.0


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("where", ["D", "E"])
def test_non_finite_input_is_reported(fresh, bad, where):
    n = 3000
    d, e = families.generate("uniform", n)
    if where == "D":
        d[1234] = bad
    else:
        e[2345] = bad
    solve(fresh, d, e)
    info, st = fresh.info_status(n)
    assert (info, st) == (-4, brdc.INTERNAL_ERROR)
    # a finite input on the same workspace afterwards
    d2, e2 = families.generate("uniform", n)
    W = solve(fresh, d2, e2).cpu().numpy()
    assert fresh.info_status(n) == (0, brdc.SUCCESS)
    ref = oracle.dstedc_dc_br(d2, e2)
    assert np.max(np.abs(W - ref)) < TOL * np.max(np.abs(ref))


def test_non_finite_input_in_a_batch(fresh):
    import torch

    off, D, E, orders, _ = families.batch(16, 17, 2000, seed=8)
    E[off[3] + 5] = np.nan
    ws = fresh.batched_workspace(off)
    fresh.dstebr_batched(off, torch.tensor(D, device="cuda"), torch.tensor(E, device="cuda"),
                         workspace=ws)
    info, st = fresh.info_status(0, ws)
    assert (info, st) == (-4, brdc.INTERNAL_ERROR)
    # the ignored E slot at the end of an instance may hold anything
    off, D, E, orders, _ = families.batch(16, 17, 2000, seed=8)
    E[off[4] - 1] = np.nan
    W = fresh.dstebr_batched(off, torch.tensor(D, device="cuda"), torch.tensor(E, device="cuda"),
                             workspace=ws).cpu().numpy()
    assert fresh.info_status(0, ws) == (0, brdc.SUCCESS)
    for b in range(len(orders)):
        lo, hi = int(off[b]), int(off[b + 1])
        ref = oracle.dstedc_dc_br(D[lo:hi], E[lo:hi - 1])
        assert np.max(np.abs(W[lo:hi] - ref)) < TOL * np.max(np.abs(ref))


def test_backward_after_a_failed_forward_does_nothing(fresh):
    """The adjoint reads the forward's checkpoints; after a non-finite input
    it returns at once with the status kept."""
    import torch

    n = 1000
    d, e = families.generate("normal", n)
    d[10] = np.nan
    ws = fresh.checkpoint_workspace(n)
    D, E = torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda")
    fresh.dstebr(D, E, workspace=ws)
    G = torch.ones(n, dtype=torch.float64, device="cuda")
    fresh.dstebr_backward(D, E, G, workspace=ws, keep_forward=True)
    assert fresh.info_status(n, ws) == (-4, brdc.INTERNAL_ERROR)
