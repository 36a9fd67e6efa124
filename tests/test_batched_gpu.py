"""Batched (forest) solves and CUDA-graph capture of the solve."""
import numpy as np
import pytest

import oracle
from brdc import families

pytestmark = pytest.mark.gpu
TOL = 1e-12


def per_instance_errors(off, W, D, E):
    errs = []
    for b in range(len(off) - 1):
        lo, hi = int(off[b]), int(off[b + 1])
        ref = oracle.dstedc_dc_br(D[lo:hi], E[lo:hi - 1])
        errs.append(float(np.max(np.abs(W[lo:hi] - ref)) / max(np.max(np.abs(ref)), 1e-300)))
    return np.array(errs)


def test_batched_mixed_orders_and_families(solver):
    import torch

    off, D, E, orders, fams = families.batch(96, 32, 3000, seed=1)
    W = solver.dstebr_batched(off, torch.tensor(D, device="cuda"),
                              torch.tensor(E, device="cuda")).cpu().numpy()
    errs = per_instance_errors(off, W, D, E)
    assert errs.max() < TOL, (errs.argmax(), errs.max())


def test_batched_includes_tiny_instances(solver):
    import torch

    orders = [1, 2, 16, 17, 5, 100, 33, 1, 64, 15]
    off = np.concatenate([[0], np.cumsum(orders)])
    rng = np.random.default_rng(9)
    D = rng.standard_normal(off[-1])
    E = rng.standard_normal(off[-1])
    for b in range(len(orders)):
        E[off[b + 1] - 1] = 7.0  # the slot between instances is ignored
    W = solver.dstebr_batched(off, torch.tensor(D, device="cuda"),
                              torch.tensor(E, device="cuda")).cpu().numpy()
    errs = per_instance_errors(off, W, D, E)
    assert errs.max() < TOL


def test_batched_agrees_with_single_solves(solver):
    # Lanes per root follow the level's K statistics, which differ between a
    # batch and a lone solve, so sums may be ordered differently: agreement
    # is to the parity tolerance, not bitwise.
    import torch

    off, D, E, orders, _ = families.batch(20, 17, 2000, seed=2)
    Wb = solver.dstebr_batched(off, torch.tensor(D, device="cuda"),
                               torch.tensor(E, device="cuda")).cpu().numpy()
    for b in range(len(orders)):
        lo, hi = int(off[b]), int(off[b + 1])
        ws = solver.dstebr(torch.tensor(D[lo:hi], device="cuda"),
                           torch.tensor(E[lo:hi - 1] if hi - lo > 1 else np.zeros(1), device="cuda"))
        w1 = ws.cpu().numpy()
        assert np.max(np.abs(w1 - Wb[lo:hi])) <= TOL * np.max(np.abs(w1))


def test_graph_capture_single_solve(solver):
    import torch

    n = 30000
    d, e = families.generate("normal", n)
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    ws = solver.workspace(n)
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        solver.set_stream(stream)
        solver.dstebr(D, E, W=W, workspace=ws)  # eager warm-up outside capture
        stream.synchronize()
        ref = W.clone()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            solver.dstebr(D, E, W=W, workspace=ws)
    torch.cuda.current_stream().wait_stream(stream)
    solver.set_stream()
    W.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(W, ref)
    # new input values flow through the captured graph
    d2, e2 = families.generate("uniform", n)
    D.copy_(torch.tensor(d2, device="cuda"))
    E.copy_(torch.tensor(e2, device="cuda"))
    g.replay()
    torch.cuda.synchronize()
    ref2 = oracle.dstedc_dc_br(d2, e2)
    assert np.max(np.abs(W.cpu().numpy() - ref2)) < TOL * np.max(np.abs(ref2))


def test_graph_capture_batched(solver):
    import torch

    off, D, E, _, _ = families.batch(64, 32, 1500, seed=3)
    Dt = torch.tensor(D, device="cuda")
    Et = torch.tensor(E, device="cuda")
    W = torch.empty(int(off[-1]), dtype=torch.float64, device="cuda")
    ws = solver.batched_workspace(off)
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        solver.set_stream(stream)
        solver.dstebr_batched(off, Dt, Et, W=W, workspace=ws)  # uploads tables
        stream.synchronize()
        ref = W.clone()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            solver.dstebr_batched(off, Dt, Et, W=W, workspace=ws)
    torch.cuda.current_stream().wait_stream(stream)
    solver.set_stream()
    W.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(W, ref)


def test_batched_workspace_reused_between_calls(solver):
    """A batched call, then other use of the same workspace bytes (a single
    solve carves them its own way; a caching allocator may hand them to
    anything), then the same batched call again: its per-instance tables
    must be rewritten, not assumed."""
    import torch

    import brdc

    off, D, E, orders, _ = families.batch(24, 17, 1500, seed=5)
    Dt = torch.tensor(D, device="cuda")
    Et = torch.tensor(E, device="cuda")
    ws = solver.batched_workspace(off)
    W0 = solver.dstebr_batched(off, Dt, Et, workspace=ws).cpu().numpy()
    assert per_instance_errors(off, W0, D, E).max() < TOL
    n = int(off[-1]) // 2
    assert brdc.workspace_size(n) <= ws.numel()
    d, e = families.generate("normal", n)
    w1 = solver.dstebr(torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda"),
                       workspace=ws).cpu().numpy()
    ref1 = oracle.dstedc_dc_br(d, e)
    assert np.max(np.abs(w1 - ref1)) < TOL * np.max(np.abs(ref1))
    W2 = solver.dstebr_batched(off, Dt, Et, workspace=ws).cpu().numpy()
    assert per_instance_errors(off, W2, D, E).max() < TOL
    ws.fill_(255)  # every byte, tables included
    W3 = solver.dstebr_batched(off, Dt, Et, workspace=ws).cpu().numpy()
    assert per_instance_errors(off, W3, D, E).max() < TOL


def test_batched_tunings_agree(solver):
    """A batch of mixed orders (tiny ones solved wholly inside the subtree
    kernel, large ones continuing with per-level kernels) gives the same
    eigenvalues whatever the subtree depth and level fusion."""
    import torch

    import brdc

    off, D, E, orders, _ = families.batch(60, 17, 3000, seed=4)
    Dt = torch.tensor(D, device="cuda")
    Et = torch.tensor(E, device="cuda")
    s = brdc.Solver()
    try:
        res = []
        for sub, fuse in ((0, 0), (0, 1 << 30), (2, 1 << 30), (4, 0), (4, 1 << 30), (5, 4096)):
            s.set_tuning(subtree_levels=sub, fused_level_rows=fuse)
            res.append(s.dstebr_batched(off, Dt, Et).cpu().numpy())
        for r in res[1:]:
            for b in range(len(orders)):
                lo, hi = int(off[b]), int(off[b + 1])
                sc = max(np.max(np.abs(res[0][lo:hi])), 1e-300)
                assert np.max(np.abs(r[lo:hi] - res[0][lo:hi])) < 1e-13 * sc, b
        errs = per_instance_errors(off, res[-1], D, E)
        assert errs.max() < TOL
    finally:
        s.close()


def test_sharded_batch_matches_whole(solver):
    """A batch split by the multi-GPU partition and solved share by share
    (here one after another on one GPU) gives the whole batch's results."""
    import torch

    from brdc.sharding import pack, partition_instances

    off, D, E, orders, _ = families.batch(40, 17, 2500, seed=6)
    whole = solver.dstebr_batched(off, torch.tensor(D, device="cuda"),
                                  torch.tensor(E, device="cuda")).cpu().numpy()
    for idx in partition_instances(orders, 3):
        o2, D2, E2 = pack(off, D, E, idx)
        part = solver.dstebr_batched(o2, torch.tensor(D2, device="cuda"),
                                     torch.tensor(E2, device="cuda")).cpu().numpy()
        for k, i in enumerate(idx):
            lo, hi = int(off[i]), int(off[i + 1])
            sc = np.max(np.abs(whole[lo:hi]))
            assert np.max(np.abs(part[o2[k]:o2[k + 1]] - whole[lo:hi])) < 1e-13 * sc
