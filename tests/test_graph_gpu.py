"""Graph replay of the plain solve (brdc_set_graphs): a call that repeats
the previous plain call's arguments is captured as a CUDA graph and
replayed.  The replay runs the same kernels on the same arguments, so its
eigenvalues are bit for bit those of ordinary launches."""
import numpy as np
import pytest

from brdc import families

pytestmark = pytest.mark.gpu


def buffers(d, e):
    import torch

    n = len(d)
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e if len(e) else np.zeros(1), device="cuda")
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    return D, E, W


@pytest.mark.parametrize("family,n", [("uniform", 65536), ("normal", 40000),
                                      ("toeplitz", 16384), ("clustered", 8192)])
def test_replay_matches_ordinary_launches(family, n):
    import brdc

    d, e = families.generate(family, n)
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e)
        ws = s.workspace(n)
        s.set_graphs(False)
        s.dstebr(D, E, W=W, workspace=ws)
        eager = W.cpu().numpy().copy()
        eager_launches = s.last_launches()
        assert not eager_launches["replayed"]
        s.set_graphs(True)
        s.dstebr(D, E, W=W, workspace=ws)  # first call of the signature: ordinary
        assert not s.last_launches()["replayed"]
        for _ in range(3):  # captured, then replayed
            W.fill_(0.0)
            s.dstebr(D, E, W=W, workspace=ws)
            rec = s.last_launches()
            assert rec["replayed"]
            assert s.info(n, ws) == 0
            assert np.array_equal(W.cpu().numpy(), eager)
            assert rec["launches"] == eager_launches["launches"]
    finally:
        s.close()


def test_new_arguments_drop_the_graph():
    import brdc
    import torch

    n = 8192
    d, e = families.generate("normal", n)
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e)
        ws = s.workspace(n)
        for _ in range(3):
            s.dstebr(D, E, W=W, workspace=ws)
        assert s.last_launches()["replayed"]
        ref = W.cpu().numpy().copy()
        W2 = torch.empty_like(W)
        s.dstebr(D, E, W=W2, workspace=ws)  # another W: ordinary launches
        assert not s.last_launches()["replayed"]
        assert np.array_equal(W2.cpu().numpy(), ref)
        # same pointers, new values: the replay reads them
        d2, e2 = families.generate("uniform", n)
        D.copy_(torch.tensor(d2))
        E.copy_(torch.tensor(e2))
        s.dstebr(D, E, W=W2, workspace=ws)
        s.dstebr(D, E, W=W2, workspace=ws)
        assert s.last_launches()["replayed"]
        plain = brdc.Solver()
        try:
            plain.set_graphs(False)
            W3 = plain.dstebr(D, E)
            assert np.array_equal(W2.cpu().numpy(), W3.cpu().numpy())
        finally:
            plain.close()
        assert not np.array_equal(W2.cpu().numpy(), ref)
    finally:
        s.close()


def test_caller_capture_uses_ordinary_launches():
    """Inside the caller's own stream capture the solve is captured as plain
    launches into the caller's graph."""
    import brdc
    import torch

    n = 16384
    d, e = families.generate("uniform", n)
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e)
        ws = s.workspace(n)
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(stream):
            s.set_stream(stream)
            s.dstebr(D, E, W=W, workspace=ws)
            s.dstebr(D, E, W=W, workspace=ws)
            stream.synchronize()
            ref = W.cpu().numpy().copy()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                s.dstebr(D, E, W=W, workspace=ws)
            W.fill_(0.0)
            g.replay()
            stream.synchronize()
            assert np.array_equal(W.cpu().numpy(), ref)
            del g
        s.set_stream(None)
    finally:
        s.close()


def test_timing_mode_uses_ordinary_launches():
    import brdc

    n = 16384
    d, e = families.generate("uniform", n)
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e)
        ws = s.workspace(n)
        for _ in range(3):
            s.dstebr(D, E, W=W, workspace=ws)
        s.set_timing(True)
        s.dstebr(D, E, W=W, workspace=ws)
        t = s.last_timings()
        assert not s.last_launches()["replayed"]
        assert t["launches"] == s.last_launches()["launches"]
        s.set_timing(False)
    finally:
        s.close()


@pytest.mark.parametrize("layout", ["pinned", "pageable", "joint"])
def test_host_entry_matches_device_entry(layout):
    """brdc_dstebr_host: the copies in, the solve and the copy out give the
    device entry's eigenvalues bit for bit, with pinned or pageable buffers;
    from the second call on the solve is a graph replay."""
    import brdc
    import torch

    n = 32768
    d, e = families.generate("normal", n)
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e)
        s.dstebr(D, E, W=W, workspace=s.workspace(n))
        ref = W.cpu().numpy().copy()
        hD = torch.tensor(d)
        hE = torch.tensor(e)
        hW = torch.empty(n, dtype=torch.float64)
        if layout == "pinned":
            hD, hE, hW = hD.pin_memory(), hE.pin_memory(), hW.pin_memory()
        elif layout == "joint":  # E right after D in one buffer: one copy in
            hDE = torch.cat([hD, hE]).pin_memory()
            hD, hE, hW = hDE[:n], hDE[n:], hW.pin_memory()
        for i in range(4):
            hW.fill_(0.0)
            s.dstebr_host(hD, hE, W=hW)
            torch.cuda.current_stream().synchronize()
            s.stream.synchronize()
            assert np.array_equal(hW.numpy(), ref)
            assert s.last_launches()["replayed"] == (i >= 1)
        # new values in the same pinned buffers reach the replay
        d2, e2 = families.generate("uniform", n)
        hD.copy_(torch.tensor(d2))
        hE.copy_(torch.tensor(e2))
        s.dstebr_host(hD, hE, W=hW)
        s.stream.synchronize()
        D.copy_(torch.tensor(d2))
        E.copy_(torch.tensor(e2))
        s.dstebr(D, E, W=W, workspace=s.workspace(n))
        assert np.array_equal(hW.numpy(), W.cpu().numpy())
    finally:
        s.close()


def test_host_entry_argument_checks():
    import brdc
    import torch

    s = brdc.Solver()
    try:
        with pytest.raises(brdc.BrdcError) as ei:
            s.dstebr_host(torch.zeros(8, dtype=torch.float64), torch.zeros(7, dtype=torch.float64),
                          workspace=torch.empty(16, dtype=torch.uint8, device="cuda"))
        assert ei.value.status == brdc.INVALID_WORKSPACE
        w = s.dstebr_host(torch.tensor([3.0], dtype=torch.float64), None)
        s.stream.synchronize()
        assert w.numpy().tolist() == [3.0]
    finally:
        s.close()


def test_replay_reports_failure_statuses():
    """The status words work in a replay as in stream launches: a NaN put
    into the same buffers between replays gives info = -4 from the replayed
    k_norm, the next clean values solve again on the same graph, and an
    iteration cap of 1 (a new signature: stream launches, then a new graph)
    reports unconverged roots."""
    import brdc
    import torch

    n = 16384
    d, e = families.generate("normal", n)
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e)
        ws = s.workspace(n)
        for _ in range(3):
            s.dstebr(D, E, W=W, workspace=ws)
        assert s.last_launches()["replayed"]
        ref = W.cpu().numpy().copy()
        D[n // 3] = float("nan")
        s.dstebr(D, E, W=W, workspace=ws)
        assert s.last_launches()["replayed"]
        assert s.info_status(n, ws) == (-4, brdc.INTERNAL_ERROR)
        D.copy_(torch.tensor(d))
        s.dstebr(D, E, W=W, workspace=ws)
        assert s.last_launches()["replayed"]
        assert s.info_status(n, ws) == (0, brdc.SUCCESS)
        assert np.array_equal(W.cpu().numpy(), ref)
        s.set_limits(secular_max_iter=1)
        for i in range(3):
            s.dstebr(D, E, W=W, workspace=ws)
            assert s.last_launches()["replayed"] == (i >= 1)
            info, st = s.info_status(n, ws)
            assert info > 0 and st == brdc.NOT_CONVERGED
        s.set_limits(secular_max_iter=64)
        s.dstebr(D, E, W=W, workspace=ws)
        assert not s.last_launches()["replayed"]
        assert np.array_equal(W.cpu().numpy(), ref)
    finally:
        s.close()


@pytest.mark.parametrize("n", [1, 2, 16, 17, 33, 1000])
def test_replay_small_orders(n):
    """Orders whose tree is one leaf, one merge or a few levels replay like
    the rest: the same bits as stream launches, call after call."""
    import brdc

    rng = np.random.default_rng(77 + n)
    d, e = rng.standard_normal(n), rng.standard_normal(max(n - 1, 1))
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e[: n - 1] if n > 1 else e)
        ws = s.workspace(n)
        s.set_graphs(False)
        s.dstebr(D, E, W=W, workspace=ws)
        ref = W.cpu().numpy().copy()
        s.set_graphs(True)
        for i in range(3):
            W.fill_(0.0)
            s.dstebr(D, E, W=W, workspace=ws)
            assert s.last_launches()["replayed"] == (i >= 1)
            assert np.array_equal(W.cpu().numpy(), ref)
    finally:
        s.close()


@pytest.mark.parametrize("keep_forward", [True, False])
def test_adjoint_replay_matches_ordinary_launches(keep_forward):
    """A loop of checkpointing forward and adjoint: both replay their graphs
    from the second step on, with gradients bit for bit those of stream
    launches."""
    import brdc
    import torch

    n = 16384
    d, e = families.generate("normal", n)
    g = np.random.default_rng(5).standard_normal(n)
    s = brdc.Solver()
    try:
        D, E, W = buffers(d, e)
        G = torch.tensor(g, device="cuda")
        gD = torch.empty(n, dtype=torch.float64, device="cuda")
        gE = torch.empty(n, dtype=torch.float64, device="cuda")
        wsc = s.new_checkpoint_workspace(n)

        def step():
            if keep_forward:
                s.dstebr(D, E, W=W, workspace=wsc)
                fwd = s.last_launches()["replayed"]
            else:
                fwd = None
            s.dstebr_backward(D, E, G, workspace=wsc, keep_forward=keep_forward, gD=gD, gE=gE)
            return fwd, s.last_launches()["replayed"]

        s.set_graphs(False)
        step()
        ref = (gD.cpu().numpy().copy(), gE.cpu().numpy()[: n - 1].copy())
        s.set_graphs(True)
        for i in range(4):
            gD.fill_(0.0)
            gE.fill_(0.0)
            fwd, bwd = step()
            assert bwd == (i >= 1)
            if keep_forward:
                assert fwd == (i >= 1)
            assert np.array_equal(gD.cpu().numpy(), ref[0])
            assert np.array_equal(gE.cpu().numpy()[: n - 1], ref[1])
    finally:
        s.close()
