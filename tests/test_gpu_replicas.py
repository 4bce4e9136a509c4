"""The weak-scaling replica path with the product in every rank: two gloo
ranks (processes) on one GPU each draw their own coupling sets
(bench.couplings, seed + rank), build the batch of every momentum sector
(bench.build_batched) and solve it, then combine their step times and work
with bench.aggregate_ranks.  The ranks' kernels never wait on one another:
the only synchronisation is the host-side gloo reduction between solves.
Every rank's energies are checked against dense FP64 diagonalisation of the
oracle's sector matrices, and the aggregate against the per-rank figures."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L, N_SETS = 10, 6


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    import qmbcuda_b200 as q
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        A = q._capi
        J, D = bench.couplings(N_SETS, rank)
        secs, b = bench.build_batched(q, L, N_SETS)
        E, summ = b.solve(J, J * D, mode=A.MODE_MIXED, max_iter=300, tol=1e-12, seed=bench.SEED)
        units = float(summ.n_products) * float(b.info.rows_total) / N_SETS
        ms, e2e, tot = bench.aggregate_ranks(torch, dist, float(summ.ms_total), 1.0 + rank, units, "cpu")
        out.put((rank, J.tolist(), D.tolist(), E.tolist(), float(summ.ms_total), units, (ms, e2e, tot)))
    finally:
        dist.destroy_process_group()


def _oracle_ground_energies(J, D):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    import qmbcuda_b200 as q
    from helpers import oracle_group, oracle_terms
    perm, ch = q.translation_group(L)
    sec = O.build_sector(oracle_group(perm, ch), L // 2)
    bonds = q.chain_bonds(L)
    txy, tz = q.xxz_terms(bonds, 1.0, 0.0), q.xxz_terms(bonds, 0.0, 1.0)
    E = np.zeros((len(J), L))
    for a in range(L):
        rows = O.active_rows(sec, a)
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(txy), a, 2 * txy.n_terms + 1)
        Axy = O.ell_to_csr(ind, val, tr, rows).toarray()
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(tz), a, 2 * tz.n_terms + 1)
        Dz = O.ell_to_csr(ind, val, tr, rows).toarray()
        H = J[:, None, None] * Axy[None] + (J * D)[:, None, None] * Dz[None]
        E[:, a] = np.linalg.eigvalsh(H)[:, 0]
    return E


def test_two_ranks_solve_their_own_coupling_sets():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    qu = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, qu)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted([qu.get(timeout=300) for _ in procs], key=lambda g: g[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert not np.allclose(got[0][1], got[1][1]), "the ranks draw different coupling sets"
    ms_max = max(g[4] for g in got)
    units_sum = sum(g[5] for g in got)
    for rank, J, D, E, ms, units, (ams, ae2e, atot) in got:
        assert ams == pytest.approx(ms_max) and ae2e == 2.0 and atot == pytest.approx(units_sum)
        e_o = _oracle_ground_energies(np.array(J), np.array(D))
        err = np.abs(np.array(E) - e_o) / np.maximum(np.abs(e_o), 1.0)
        assert err.max() <= 1e-10, (rank, err.max())
