"""The multi-rank bench path on CPU: two gloo ranks solve disjoint coupling
sets (seed + rank), the whole-job step time is the maximum over ranks and the
work is the sum over ranks."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        J, D = bench.couplings(8, rank)
        ms = 10.0 + 5.0 * rank
        e2e = 1.0 + rank
        units = 100.0 * (rank + 1)
        res = bench.aggregate_ranks(torch, dist, ms, e2e, units, "cpu")
        out.put((rank, res, J.tolist(), D.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_max_time_and_summed_work():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got.sort()
    for rank, (ms, e2e, units), J, D in got:
        assert ms == 15.0 and e2e == 2.0 and units == 300.0
    # the two ranks draw different coupling sets
    assert not np.allclose(got[0][2], got[1][2])
    assert all(0.5 <= j <= 1.5 for j in got[0][2] + got[1][2])
    assert all(0.0 <= d <= 2.0 for d in got[0][3] + got[1][3])


def test_single_process_aggregate_is_identity():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_ranks(torch, None, 3.0, 4.0, 5.0, "cpu") == (3.0, 4.0, 5.0)
