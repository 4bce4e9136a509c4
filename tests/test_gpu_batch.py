"""Batched Lanczos (many coupling sets x many momentum sectors) against
single-sector FP64 solves and dense FP64 diagonalisation."""
import numpy as np
import pytest

import oracle as O
import qmbcuda_b200 as q
from helpers import oracle_group, oracle_terms

pytestmark = pytest.mark.gpu
A = q._capi


def _sectors(L):
    perm, ch = q.translation_group(L)
    return [q.Sector(L, L // 2, perm).set_irrep(ch[a]) for a in range(L)], perm, ch


@pytest.mark.parametrize("mode", [A.MODE_FP64, A.MODE_MIXED])
def test_batch_matches_single_solves(mode):
    L, n_sets = 10, 40
    secs, perm, ch = _sectors(L)
    bonds = q.chain_bonds(L)
    b = q.Batch(secs, q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"), n_sets)
    rng = np.random.default_rng(20261203)
    delta = rng.uniform(0, 2, n_sets)
    J = rng.uniform(0.5, 1.5, n_sets)
    E, summ = b.solve(J, J * delta, mode=mode, max_iter=200, tol=1e-12)
    assert E.shape == (n_sets, L)
    for i in (0, 7, n_sets - 1):
        for a in (0, 3, 5):
            t = q.xxz_terms(bonds, J[i], J[i] * delta[i])
            e1 = q.Hamiltonian(secs[a], t).lanczos(tol=1e-12).E0
            assert abs(E[i, a] - e1) <= 1e-10 * abs(e1), (i, a, E[i, a], e1)


def test_batch_dense_oracle_and_hv():
    import torch
    L, n_sets = 8, 32
    secs, perm, ch = _sectors(L)
    bonds = q.chain_bonds(L)
    txy, tz = q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z")
    b = q.Batch(secs, txy, tz, n_sets)
    J = np.linspace(0.5, 1.5, n_sets)
    D = np.linspace(0.0, 2.0, n_sets)
    E, _ = b.solve(J, J * D, mode=A.MODE_FP64, tol=1e-12)
    g = oracle_group(perm, ch)
    sec = O.build_sector(g, L // 2)
    for i in (0, 13, 31):
        for a in range(L):
            t = q.xxz_terms(bonds, J[i], J[i] * D[i])
            rc, ind, val, tr = O.ell_terms(sec, oracle_terms(t), a, 2 * t.n_terms + 1)
            rows = O.active_rows(sec, a)
            if len(rows) == 0:
                continue
            e = O.ground_energy_dense(O.ell_to_csr(ind, val, tr, rows))
            assert abs(E[i, a] - e) <= 1e-10 * max(1.0, abs(e))
    # one batched H*v in FP64 against per-sector products
    info = b.info
    off, cp = b.layout()
    tot = int(off[-1])
    x = torch.randn(tot, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    b.hv_dev(x.data_ptr(), y.data_ptr(), A.PREC_FP64)
    torch.cuda.synchronize()
    xs, ys = x.cpu().numpy(), y.cpu().numpy()
    stride = info.set_stride
    for a in (0, 2):
        rows = O.active_rows(sec, a)
        t = q.xxz_terms(bonds, 1.0, 0.0)
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(t), a, 2 * t.n_terms + 1)
        M = O.ell_to_csr(ind, val, tr, rows)
        tz1 = q.xxz_terms(bonds, 0.0, 1.0)
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(tz1), a, 2 * tz1.n_terms + 1)
        Dz = O.ell_to_csr(ind, val, tr, rows)
        n = len(rows)
        o = int(off[a])
        if cp[a]:
            xv = xs[o:o + 2 * n * stride].view(np.complex128).reshape(n, stride)
            yv = ys[o:o + 2 * n * stride].view(np.complex128).reshape(n, stride)
        else:
            xv = xs[o:o + n * stride].reshape(n, stride)
            yv = ys[o:o + n * stride].reshape(n, stride)
        for i in (0, 5):
            want = J[i] * (M @ xv[:, i]) + J[i] * D[i] * (Dz @ xv[:, i])
            np.testing.assert_allclose(yv[:, i], want, atol=1e-11 * np.abs(want).max())


@pytest.mark.parametrize("mode", [A.MODE_FP64, A.MODE_MIXED, A.MODE_FP32])
def test_batch_many_sets_dense_oracle(mode):
    """200 coupling sets x 12 sectors: convergence spreads over many steps,
    so the unconverged tail continues in a compacted sub-batch.  Every
    energy is checked against dense diagonalisation of its sector matrix."""
    L, n_sets = 12, 200
    secs, perm, ch = _sectors(L)
    bonds = q.chain_bonds(L)
    b = q.Batch(secs, q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"), n_sets)
    rng = np.random.default_rng(7)
    D = rng.uniform(0, 2, n_sets)
    J = rng.uniform(0.5, 1.5, n_sets)
    E, summ = b.solve(J, J * D, mode=mode, max_iter=300, tol=1e-12)
    g = oracle_group(perm, ch)
    sec = O.build_sector(g, L // 2)
    txy, tz = q.xxz_terms(bonds, 1.0, 0.0), q.xxz_terms(bonds, 0.0, 1.0)
    tol = 1e-5 if mode == A.MODE_FP32 else 1e-10
    for a in range(L):
        rows = O.active_rows(sec, a)
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(txy), a, 2 * txy.n_terms + 1)
        Axy = O.ell_to_csr(ind, val, tr, rows).toarray()
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(tz), a, 2 * tz.n_terms + 1)
        Dz = O.ell_to_csr(ind, val, tr, rows).toarray()
        H = J[:, None, None] * Axy[None] + (J * D)[:, None, None] * Dz[None]
        e = np.linalg.eigvalsh(H)[:, 0]
        err = np.abs(E[:, a] - e) / np.maximum(np.abs(e), 1.0)
        assert err.max() <= tol, (a, err.max(), int(err.argmax()))


def test_batch_compaction_levels(monkeypatch):
    """With QMB_SUB_COMPACT_RATIO=0.9 the unconverged problems of a compacted
    sub-batch move on into smaller ones (up to three levels); every energy
    still equals dense diagonalisation of its sector matrix, in FP64 and in
    mixed mode."""
    monkeypatch.setenv("QMB_SUB_COMPACT_RATIO", "0.9")
    L, n_sets = 12, 200
    secs, perm, ch = _sectors(L)
    bonds = q.chain_bonds(L)
    b = q.Batch(secs, q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"), n_sets)
    rng = np.random.default_rng(17)
    D = rng.uniform(0, 2, n_sets)
    J = rng.uniform(0.5, 1.5, n_sets)
    g = oracle_group(perm, ch)
    sec = O.build_sector(g, L // 2)
    txy, tz = q.xxz_terms(bonds, 1.0, 0.0), q.xxz_terms(bonds, 0.0, 1.0)
    e = np.zeros((n_sets, L))
    for a in range(L):
        rows = O.active_rows(sec, a)
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(txy), a, 2 * txy.n_terms + 1)
        Axy = O.ell_to_csr(ind, val, tr, rows).toarray()
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(tz), a, 2 * tz.n_terms + 1)
        Dz = O.ell_to_csr(ind, val, tr, rows).toarray()
        H = J[:, None, None] * Axy[None] + (J * D)[:, None, None] * Dz[None]
        e[:, a] = np.linalg.eigvalsh(H)[:, 0]
    for mode in (A.MODE_FP64, A.MODE_MIXED):
        E, summ = b.solve(J, J * D, mode=mode, max_iter=300, tol=1e-12)
        err = np.abs(E - e) / np.maximum(np.abs(e), 1.0)
        assert err.max() <= 1e-10, (mode, err.max())


def test_batch_ring_growth_bit_identical(monkeypatch):
    """A Krylov ring that starts at 4 vectors doubles until the FP32 phase
    fits: the solve is bit-identical to one whose ring held the phase from
    the start, and the ring ends no larger than its growth needed."""
    L, n_sets = 10, 40
    bonds = q.chain_bonds(L)
    rng = np.random.default_rng(11)
    D = rng.uniform(0, 2, n_sets)
    J = rng.uniform(0.5, 1.5, n_sets)
    out = []
    for start in (None, "4"):
        if start is None:
            monkeypatch.delenv("QMB_RING_START", raising=False)
        else:
            monkeypatch.setenv("QMB_RING_START", start)
        secs, perm, ch = _sectors(L)
        b = q.Batch(secs, q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"),
                    n_sets)
        E, r = b.solve(J, J * D, mode=A.MODE_MIXED, max_iter=300, tol=1e-12)
        out.append((E, r.iters, r.iters_low, list(b.info.ring_slots)))
        b.close()
    (E0, it0, lo0, ring0), (E1, it1, lo1, ring1) = out
    assert np.array_equal(E0.view(np.uint64), E1.view(np.uint64))
    assert (it0, lo0) == (it1, lo1)
    assert min(ring0) >= 128
    # grown from 4 by doubling; the longer FP32 phase (iters_low steps) fits
    assert all(s in (4, 8, 16, 32, 64, 128, 256) for s in ring1), ring1
    assert max(ring1) >= lo1 + 1 and max(ring1) <= 2 * (lo1 + 10), (ring1, lo1)


@pytest.mark.parametrize("mode", [A.MODE_FP64, A.MODE_MIXED])
def test_host_loop_matches_device_loop(mode, monkeypatch):
    """QMB_HOST_LOOP=1 launches the device loops' blocks from the host (for
    profilers, which do not see inside conditional graphs): the same kernels
    in the same order, so the energies are bit-identical, with and without
    the compacted tail (200 sets spread the convergence steps)."""
    L, n_sets = 12, 200
    bonds = q.chain_bonds(L)
    rng = np.random.default_rng(7)
    D = rng.uniform(0, 2, n_sets)
    J = rng.uniform(0.5, 1.5, n_sets)
    out = []
    for host in (None, "1"):
        if host is None:
            monkeypatch.delenv("QMB_HOST_LOOP", raising=False)
        else:
            monkeypatch.setenv("QMB_HOST_LOOP", host)
        secs, perm, ch = _sectors(L)
        b = q.Batch(secs, q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"),
                    n_sets)
        E, r = b.solve(J, J * D, mode=mode, max_iter=300, tol=1e-12, seed=5)
        out.append((E, r.iters, r.iters_low, r.n_products))
        b.close()
    (E0, it0, lo0, p0), (E1, it1, lo1, p1) = out
    assert np.array_equal(E0.view(np.uint64), E1.view(np.uint64))
    assert (it0, lo0, p0) == (it1, lo1, p1)


def test_batch_real_sectors_alone_and_in_complex_kind():
    """Real sectors form their own kind when the batch has no complex ones,
    and join the complex kind when they are a small part of it (L=12: two
    real momenta of twelve).  Both give the single-sector FP64 energies."""
    L, n_sets = 12, 16
    secs, perm, ch = _sectors(L)
    bonds = q.chain_bonds(L)
    txy, tz = q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z")
    J = np.linspace(0.6, 1.4, n_sets)
    D = np.linspace(0.1, 1.9, n_sets)
    real = [secs[0], secs[L // 2]]
    b_real = q.Batch(real, txy, tz, n_sets)
    b_all = q.Batch(secs, txy, tz, n_sets)
    assert list(b_real.layout()[1]) == [0, 0]
    cp_all = b_all.layout()[1]
    assert cp_all[0] == 1 and cp_all[L // 2] == 1 and all(cp_all)
    for mode in (A.MODE_FP64, A.MODE_MIXED):
        E_real, _ = b_real.solve(J, J * D, mode=mode, max_iter=300, tol=1e-12)
        E_all, _ = b_all.solve(J, J * D, mode=mode, max_iter=300, tol=1e-12)
        for i in (0, 9, n_sets - 1):
            for col, a in ((0, 0), (1, L // 2)):
                t = q.xxz_terms(bonds, J[i], J[i] * D[i])
                e1 = q.Hamiltonian(secs[a], t).lanczos(tol=1e-12).E0
                assert abs(E_real[i, col] - e1) <= 1e-10 * abs(e1), (mode, i, a)
                assert abs(E_all[i, a] - e1) <= 1e-10 * abs(e1), (mode, i, a)


def test_mixed_restart_near_degenerate_pair():
    """L=20 XXZ chain at Delta = 7.2e-5, k = pi: the two lowest levels are
    1.2e-7 |E| apart, below what the FP32 phase separates.  With 256 start
    vectors (one per coupling set, all sets equal) the mixed solve must end
    on the ground level for all but the starts whose FP32 vector holds
    almost none of it, and never further off than the splitting.  FP64 mode
    has the same exposure for starts that hold almost none of the ground
    level, so it is held to the splitting bound only."""
    L, n_sets = 20, 256
    J0, D = 1.0086762452351132, 7.209233047955621e-05
    perm, ch = q.translation_group(L)
    bonds = q.chain_bonds(L)
    s = q.Sector(L, L // 2, perm).set_irrep(ch[L // 2])
    e_ref = q.Hamiltonian(s, q.xxz_terms(bonds, J0, J0 * D)).lanczos(
        mode=A.MODE_FP64, tol=1e-14, max_iter=600, reorth=2).E0
    b = q.Batch([s], q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"), n_sets)
    J, JD = np.full(n_sets, J0), np.full(n_sets, J0 * D)
    split = 1.2e-7
    E64, _ = b.solve(J, JD, mode=A.MODE_FP64, max_iter=300, tol=1e-12)
    err64 = np.abs(E64[:, 0] - e_ref) / abs(e_ref)
    assert err64.max() <= split
    Em, _ = b.solve(J, JD, mode=A.MODE_MIXED, max_iter=300, tol=1e-12)
    err = np.abs(Em[:, 0] - e_ref) / abs(e_ref)
    assert err.max() <= split
    # without the gap cap 126 of the 256 starts end on the upper level, with
    # the default cap 8 did in one run
    assert (err > 1e-9).sum() <= 48, int((err > 1e-9).sum())


@pytest.mark.parametrize("variant", range(8))
def test_every_product_variant_matches_the_oracle(variant, monkeypatch):
    """Each batched-product variant the tuner may choose (QMB_BHV_VARIANT
    fixes it): one FP64 and one FP32 product on 256 coupling sets against the
    oracle's sector matrices, and a mixed and an FP64 batched solve against
    dense FP64 energies."""
    import torch
    monkeypatch.setenv("QMB_BHV_VARIANT", str(variant))
    L, n_sets = 12, 256
    secs, perm, ch = _sectors(L)
    bonds = q.chain_bonds(L)
    b = q.Batch(secs, q.xxz_terms(bonds, 1.0, 0.0, part="xy"), q.xxz_terms(bonds, 0.0, 1.0, part="z"), n_sets)
    rng = np.random.default_rng(variant)
    J = rng.uniform(0.5, 1.5, n_sets)
    D = rng.uniform(0.0, 2.0, n_sets)
    E64, _ = b.solve(J, J * D, mode=A.MODE_FP64, tol=1e-12)
    Emx, _ = b.solve(J, J * D, mode=A.MODE_MIXED, tol=1e-12)
    assert b.info.variant_fp64 == variant and b.info.variant_fp32 == variant
    g = oracle_group(perm, ch)
    sec = O.build_sector(g, L // 2)
    mats = {}
    for a in range(L):
        rows = O.active_rows(sec, a)
        txy = q.xxz_terms(bonds, 1.0, 0.0)
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(txy), a, 2 * txy.n_terms + 1)
        Mxy = O.ell_to_csr(ind, val, tr, rows)
        tz = q.xxz_terms(bonds, 0.0, 1.0)
        rc, ind, val, tr = O.ell_terms(sec, oracle_terms(tz), a, 2 * tz.n_terms + 1)
        mats[a] = (Mxy, O.ell_to_csr(ind, val, tr, rows))
    for i in (0, 101, 255):
        for a in (0, 1, L // 2, L - 1):
            Mxy, Mz = mats[a]
            e = O.ground_energy_dense(J[i] * Mxy + J[i] * D[i] * Mz)
            assert abs(E64[i, a] - e) <= 1e-10 * abs(e), (i, a, E64[i, a], e)
            assert abs(Emx[i, a] - e) <= 1e-10 * abs(e), (i, a, Emx[i, a], e)
    off, cp = b.layout()
    tot = int(off[-1])
    stride = b.info.set_stride
    for prec, dt, tol in ((A.PREC_FP64, torch.float64, 1e-12), (A.PREC_FP32, torch.float32, 2e-6)):
        x = torch.randn(tot, dtype=dt, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
        y = torch.zeros_like(x)
        b.hv_dev(x.data_ptr(), y.data_ptr(), prec)
        torch.cuda.synchronize()
        xs, ys = x.double().cpu().numpy(), y.double().cpu().numpy()
        for a in (0, 1, L // 2):
            Mxy, Mz = mats[a]
            n = Mxy.shape[0]
            o = int(off[a])
            if cp[a]:
                xv = (xs[o:o + 2 * n * stride:2] + 1j * xs[o + 1:o + 2 * n * stride:2]).reshape(n, stride)
                yv = (ys[o:o + 2 * n * stride:2] + 1j * ys[o + 1:o + 2 * n * stride:2]).reshape(n, stride)
            else:
                xv = xs[o:o + n * stride].reshape(n, stride)
                yv = ys[o:o + n * stride].reshape(n, stride)
            for i in (0, 77, 255):
                want = J[i] * (Mxy @ xv[:, i]) + J[i] * D[i] * (Mz @ xv[:, i])
                np.testing.assert_allclose(yv[:, i], want, rtol=0, atol=tol * np.abs(want).max())
    b.close()
