"""The host side of sharded solves on the CPU: the index ranges of the ranks and the
all-gather over torch.distributed (gloo, world size 2), which must deliver every rank's row
in rank order: the fold of the rank rows (pass_fold in csrc/reduce.cuh) relies on it."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "lbfgsb-gpu_b200")


def test_shard_ranges_tile():
    sys.path.insert(0, PKG)
    import lbfgsb_b200 as LB
    for n, world in [(16, 2), (1024, 3), (7, 7), (4097, 8), (16777216, 8)]:
        rs = LB.shard_ranges(n, world)
        assert len(rs) == world
        assert rs[0][0] == 0
        for (o1, s1), (o2, _) in zip(rs, rs[1:]):
            assert o2 == o1 + s1
        assert rs[-1][0] + rs[-1][1] == n
        sizes = [s for _, s in rs]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import ctypes as C
    import torch.distributed as dist
    sys.path.insert(0, PKG)
    import lbfgsb_b200 as LB
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        ag = LB.DistAllGather(device=False)
        cb = ag.callback()
        fn = C.cast(cb, C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p))
        out = []
        for count in (1, 3, 256):
            send = np.arange(count, dtype=np.float64) + 1000.0 * rank
            recv = np.full(world * count, np.nan)
            rc = fn(None, send.ctypes.data, recv.ctypes.data, count, None)
            out.append((rc, recv.tolist()))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_allgather_rank_order_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank in range(2):
        for (rc, recv), count in zip(got[rank], (1, 3, 256)):
            assert rc == 0
            want = np.concatenate([np.arange(count) + 1000.0 * r for r in range(2)])
            assert np.array_equal(np.array(recv), want)
