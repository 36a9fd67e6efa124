"""Host logic of multi-GPU runs, on CPU: the batch partition and the
max-over-ranks timing of the bench, the latter with two gloo ranks."""
import os
import socket

import numpy as np
import pytest

from brdc import families
from brdc.sharding import max_over_ranks, pack, partition_instances


def test_partition_covers_and_balances():
    orders = families.batch_orders(500, 32, 8192, seed=3)
    for world in (1, 2, 3, 8):
        parts = partition_instances(orders, world)
        assert len(parts) == world
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(orders)))
        loads = [float(np.sum(orders[p].astype(float) ** 2)) for p in parts]
        # LPT is within 4/3 of the optimum; against the mean it is close
        assert max(loads) <= 1.05 * np.mean(loads) + float(np.max(orders)) ** 2
        assert partition_instances(orders, world)[0].tolist() == parts[0].tolist()


def test_pack_roundtrip():
    off, D, E, orders, _ = families.batch(20, 17, 300, seed=1)
    idx = [3, 7, 11]
    o2, D2, E2 = pack(off, D, E, idx)
    for k, i in enumerate(idx):
        lo, hi = int(off[i]), int(off[i + 1])
        assert np.array_equal(D2[o2[k]:o2[k + 1]], D[lo:hi])
        assert np.array_equal(E2[o2[k]:o2[k + 1] - 1], E[lo:hi - 1])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        v = max_over_ranks(1.5 + rank, dist)
        out.put((rank, v))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 2.5, 1: 2.5}


def test_max_over_ranks_single():
    assert max_over_ranks(3.0, None) == 3.0
