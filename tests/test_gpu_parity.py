"""GPU parity: tables, matrices and H*v through the C ABI against the oracle.

Bit-exact for integer tables (representatives, orbit map, ELL indices and row
counts); FP64 values within 1e-13 absolute; FP32 within 2e-6 relative.
"""
import numpy as np
import pytest

import oracle as O
import qmbcuda_b200 as q
from helpers import oracle_group, oracle_terms, sector_cases

pytestmark = pytest.mark.gpu

CASES = sector_cases()
IDS = [c[0] for c in CASES]


def _irreps(chars):
    n = chars.shape[0]
    return sorted(set([0, n // 2, n - 1, 1 % n]))


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_representatives_norms_orbit_map(case):
    name, L, k, perm, chars, flip, _ = case
    g = oracle_group(perm, chars, flip)
    sec_o = O.build_sector(g, k)
    s = q.Sector(L, k, perm, spin_flip=flip)
    info = s.info
    assert info.n_states == O.binom(L, k)
    reps = s.reps()
    assert np.array_equal(reps, sec_o.reps)
    assert np.array_equal(s.orbit_map(), sec_o.orbit)
    for a in _irreps(chars):
        s.set_irrep(chars[a])
        nrm = s.norms()
        # non-null orbits to 1e-13; null ones are round-off zeros on both sides
        live = sec_o.norms[:, a] >= 1e-6
        np.testing.assert_allclose(nrm[live], sec_o.norms[live, a], rtol=0, atol=1e-13)
        assert (nrm[~live] < 1e-6).all()
        act = s.active()
        assert np.array_equal(act, O.active_rows(sec_o, a))


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_lookup(case):
    name, L, k, perm, chars, flip, _ = case
    s = q.Sector(L, k, perm, spin_flip=flip)
    reps = s.reps()
    rng = np.random.default_rng(7)
    states = O.enumerate_sector(L, k)
    pick = states[rng.integers(0, len(states), 500)]
    orb, el = s.lookup(pick)
    g = oracle_group(perm, chars, flip)
    for t, o, e in zip(pick, orb, el):
        assert o >= 0
        r = reps[o]
        z, gi = divmod(int(e), g.G)
        assert O.lib().oc_apply(int(t), L, np.ascontiguousarray(g.perm[gi]), z) == r
    bad = np.array([0, (1 << L) - 1, 1], np.uint64)
    orb, _ = s.lookup(bad)
    assert (orb[[0, 1]] == -1).all()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_ell_reference_layout(case):
    name, L, k, perm, chars, flip, bonds = case
    terms = q.xxz_terms(bonds, 1.0 + 0.25j if "chain12_T" == name else 1.0, 0.7)
    g = oracle_group(perm, chars, flip)
    sec_o = O.build_sector(g, k)
    s = q.Sector(L, k, perm, spin_flip=flip)
    W = 2 * len(bonds) + 1
    for a in _irreps(chars):
        s.set_irrep(chars[a])
        ind, val, tr = q.export_ref(s, terms, W)
        rc, ind_o, val_o, tr_o = O.ell_terms(sec_o, oracle_terms(terms), a, W)
        assert rc >= 0
        assert np.array_equal(tr, tr_o)
        # compare used slots only (unused ones are zero on both sides)
        assert np.array_equal(ind, ind_o)
        np.testing.assert_allclose(val, val_o, rtol=0, atol=1e-13)


def test_ell_overflow_is_an_error():
    p, ch = q.translation_group(10)
    s = q.Sector(10, 5, p).set_irrep(ch[0])
    with pytest.raises(q.QMBError) as e:
        q.export_ref(s, q.xxz_terms(q.chain_bonds(10), 1.0, 1.0), 3)
    assert e.value.status == q._capi.QMB_ERR_ELL_OVERFLOW


def test_nosym_layout_matches_reference_rule():
    L, k = 10, 5
    bonds = q.chain_bonds(L)
    # T_standard-style pair list with unequal weights to exercise the swap
    ti = np.array([i for i, j in bonds] + [j for i, j in bonds], np.int32)
    tj = np.array([j for i, j in bonds] + [i for i, j in bonds], np.int32)
    tv = np.ones(len(ti), np.complex128) * 0.8
    cap = 4 * len(ti)
    n_ops = np.zeros(cap, np.int32); codes = np.zeros(2 * cap, np.int32)
    sites = np.zeros(2 * cap, np.int32); sc = np.zeros(2 * cap); nt = q._capi.C.c_int()
    P = q._capi.ptr
    q.check(q.lib().qmb_terms_from_pairs(len(ti), P(ti), P(tj), P(q._capi.cplx_buf(tv)), 1.0, 0.5, 1,
                                         cap, P(n_ops), P(codes), P(sites), P(sc), q._capi.C.byref(nt)))
    n = nt.value
    t = q.TermTable(n_ops[:n], codes[:2 * n].reshape(n, 2), sites[:2 * n].reshape(n, 2),
                    sc[:2 * n].view(np.complex128))
    W = 12
    ind, val, tr = q.export_nosym(L, k, t, W)
    rc, ind_o, val_o, tr_o = O.ell_nosym(L, k, ti, tj, tv, 1.0, 0.5, W)
    assert rc >= 0
    assert np.array_equal(tr, tr_o) and np.array_equal(ind, ind_o)
    np.testing.assert_allclose(val, val_o, atol=1e-14)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_hv_stored_and_matrix_free(case):
    name, L, k, perm, chars, flip, bonds = case
    terms = q.xxz_terms(bonds, 1.0, 0.5)
    g = oracle_group(perm, chars, flip)
    sec_o = O.build_sector(g, k)
    s = q.Sector(L, k, perm, spin_flip=flip)
    a = 1 % chars.shape[0]
    s.set_irrep(chars[a])
    if s.info.n_active == 0:
        pytest.skip("empty irrep")
    h = q.Hamiltonian(s, terms)
    W = 2 * len(bonds) + 1
    rc, ind_o, val_o, tr_o = O.ell_terms(sec_o, oracle_terms(terms), a, W)
    A = O.ell_to_csr(ind_o, val_o, tr_o, O.active_rows(sec_o, a))
    n = A.shape[0]
    assert h.info.n_rows == n
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n) + (1j * rng.standard_normal(n) if h.info.is_complex else 0)
    y_o = A @ x
    y = h.hv_host(x, q._capi.PREC_FP64)
    np.testing.assert_allclose(y, y_o, rtol=0, atol=1e-12 * np.abs(y_o).max())
    y32 = h.hv_host(x, q._capi.PREC_FP32)
    np.testing.assert_allclose(y32, y_o, rtol=0, atol=2e-6 * np.abs(y_o).max())
    import torch
    dt = torch.complex128 if h.info.is_complex else torch.float64
    xd = torch.tensor(x, dtype=dt, device="cuda")
    yd = torch.zeros_like(xd)
    h.hv_dev(xd.data_ptr(), yd.data_ptr(), q._capi.PREC_FP64, matrix_free=True)
    torch.cuda.synchronize()
    np.testing.assert_allclose(yd.cpu().numpy(), y_o, rtol=0, atol=1e-12 * np.abs(y_o).max())


@pytest.mark.parametrize("L,k,flip,a", [(12, 6, False, 0), (12, 6, False, 1), (16, 8, True, 3),
                                         (32, 4, False, 0), (32, 4, False, 1), (36, 3, False, 0),
                                         (36, 3, False, 1), (34, 4, False, 11)],
                         ids=lambda v: str(v))
def test_matrix_free_active_lookup(L, k, flip, a, monkeypatch):
    """The matrix-free operator's row lookup over the active orbits: 32-bit
    representatives up to L = 32 (the run-candidate orbit minimum of full
    rotation groups, funnel shifts at L = 32), 64-bit beyond; the sector's
    tables when every orbit is active, its own bucket table when some orbits
    are null; beyond 32 sites the hash table as well (forced here with
    QMB_MF_HASH=1, including its misses on null orbits).  FP64 and FP32
    products against the oracle's matrix with each lookup (per-lane hash,
    per-lane bucket search, warp-cooperative), and a matrix-free FP64 solve
    against the stored one."""
    import torch
    perm, ch = q.translation_group(L)
    chars = np.block([[ch, ch], [ch, -ch]]) if flip else ch
    terms = q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), [1.0] * L + [0.3] * L, 0.7)
    sec_o = O.build_sector(oracle_group(perm, chars, flip), k)
    s = q.Sector(L, k, perm, spin_flip=flip).set_irrep(chars[a])
    act = O.active_rows(sec_o, a)
    assert (len(act) < sec_o.R) == (a != 0), "the cases cover both table forms"
    h = q.Hamiltonian(s, terms)
    W = 4 * L + 1
    rc, ind_o, val_o, tr_o = O.ell_terms(sec_o, oracle_terms(terms), a, W)
    assert rc >= 0
    A = O.ell_to_csr(ind_o, val_o, tr_o, act)
    n = A.shape[0]
    assert h.info.n_rows == n
    rng = np.random.default_rng(L + a)
    x = rng.standard_normal(n) + (1j * rng.standard_normal(n) if h.info.is_complex else 0)
    y_o = A @ x
    # beyond 32 sites the handle also gets the hash table (forced at this
    # size), searched by default; QMB_MF_HASH=0 searches the bucket table
    monkeypatch.setenv("QMB_MF_HASH", "1")
    for lookup, hash_env in (("lane", "1"), ("lane", "0"), ("warp", "1")):
        monkeypatch.setenv("QMB_MF_LOOKUP", lookup)
        monkeypatch.setenv("QMB_MF_HASH", hash_env)
        for prec, tol in ((q._capi.PREC_FP64, 1e-12), (q._capi.PREC_FP32, 2e-6)):
            if prec == q._capi.PREC_FP64:
                dt = torch.complex128 if h.info.is_complex else torch.float64
            else:
                dt = torch.complex64 if h.info.is_complex else torch.float32
            xd = torch.tensor(x, dtype=dt, device="cuda")
            yd = torch.zeros_like(xd)
            h.hv_dev(xd.data_ptr(), yd.data_ptr(), prec, matrix_free=True)
            torch.cuda.synchronize()
            np.testing.assert_allclose(yd.cpu().numpy(), y_o, rtol=0, atol=tol * np.abs(y_o).max())
    monkeypatch.delenv("QMB_MF_LOOKUP")
    monkeypatch.delenv("QMB_MF_HASH")
    A64 = q._capi
    r_st = h.lanczos(mode=A64.MODE_FP64, tol=1e-12)
    r_mf = h.lanczos(mode=A64.MODE_FP64, tol=1e-12, hv=A64.HV_MATRIX_FREE)
    assert abs(r_mf.E0 - r_st.E0) <= 1e-10 * abs(r_st.E0)


@pytest.mark.parametrize("nx,ny,flip", [(3, 4, True), (4, 3, False), (6, 2, True), (2, 5, True), (4, 4, True)],
                         ids=lambda v: str(v))
def test_torus_orbit_search(nx, ny, flip):
    """The row-candidate orbit minimum of torus translation groups (with and
    without spin inversion, rows of 2 to 6 sites): representatives and the
    orbit map bit-exact against the oracle's full search, and the stored and
    matrix-free FP64 products against the oracle's matrix."""
    import torch
    perm, ch = q.translation_group(nx, ny)
    L = nx * ny
    k = L // 2
    chars = np.block([[ch, ch], [ch, -ch]]) if flip else ch
    g = oracle_group(perm, chars, flip)
    sec_o = O.build_sector(g, k)
    s = q.Sector(L, k, perm, spin_flip=flip)
    assert np.array_equal(s.reps(), sec_o.reps)
    assert np.array_equal(s.orbit_map(), sec_o.orbit)
    a = 1 % chars.shape[0]
    s.set_irrep(chars[a])
    terms = q.xxz_terms(q.square_bonds(nx, ny), 1.0, 0.6)
    h = q.Hamiltonian(s, terms)
    W = 2 * len(q.square_bonds(nx, ny)) + 1
    rc, ind_o, val_o, tr_o = O.ell_terms(sec_o, oracle_terms(terms), a, W)
    assert rc >= 0
    A = O.ell_to_csr(ind_o, val_o, tr_o, O.active_rows(sec_o, a))
    n = A.shape[0]
    assert h.info.n_rows == n
    rng = np.random.default_rng(nx * 10 + ny)
    x = rng.standard_normal(n) + (1j * rng.standard_normal(n) if h.info.is_complex else 0)
    y_o = A @ x
    np.testing.assert_allclose(h.hv_host(x, q._capi.PREC_FP64), y_o, rtol=0, atol=1e-12 * np.abs(y_o).max())
    dt = torch.complex128 if h.info.is_complex else torch.float64
    xd = torch.tensor(x, dtype=dt, device="cuda")
    yd = torch.zeros_like(xd)
    h.hv_dev(xd.data_ptr(), yd.data_ptr(), q._capi.PREC_FP64, matrix_free=True)
    torch.cuda.synchronize()
    np.testing.assert_allclose(yd.cpu().numpy(), y_o, rtol=0, atol=1e-12 * np.abs(y_o).max())


def test_single_block_coded_layout(monkeypatch):
    """A matrix whose vectors fit L2 but whose FP32 entry stream exceeds
    256 MB (L=30 J1-J2, k=0 even: 2.6 M rows) gets the coded layout with one
    column block (32-bit entries: an 8-bit value code above the column), for
    its FP32 and its FP64 values: the products equal the plain sliced-ELL
    products to FP32 / FP64 rounding, and a mixed solve on it equals the FP64
    energy."""
    import torch
    L = 30
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    terms = q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), [1.0] * L + [0.45] * L, [0.9] * L + [0.4] * L)
    h = q.Hamiltonian(s, terms)
    assert h.info.coded == 1 and h.info.coded_fp64 == 1
    monkeypatch.setenv("QMB_COLUMN_BLOCKS", "0")
    hp = q.Hamiltonian(s, terms)
    assert hp.info.coded == 0 and hp.info.coded_fp64 == 0
    n = int(h.info.n_rows)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(n, dtype=torch.float32, device="cuda", generator=g)
    y1, y2 = torch.empty_like(x), torch.empty_like(x)
    h.hv_dev(x.data_ptr(), y1.data_ptr(), q._capi.PREC_FP32)
    hp.hv_dev(x.data_ptr(), y2.data_ptr(), q._capi.PREC_FP32)
    torch.cuda.synchronize()
    assert float((y1 - y2).abs().max()) <= 2e-6 * float(y2.abs().max())
    # the FP64 values coded the same way: the products agree to FP64 rounding
    x64 = x.double()
    z1, z2 = torch.empty_like(x64), torch.empty_like(x64)
    h.hv_dev(x64.data_ptr(), z1.data_ptr(), q._capi.PREC_FP64)
    hp.hv_dev(x64.data_ptr(), z2.data_ptr(), q._capi.PREC_FP64)
    torch.cuda.synchronize()
    assert float((z1 - z2).abs().max()) <= 1e-13 * float(z2.abs().max())
    A = q._capi
    r64 = h.lanczos(mode=A.MODE_FP64, tol=1e-12)
    rmx = h.lanczos(mode=A.MODE_MIXED, tol=1e-12)
    assert abs(rmx.E0 - r64.E0) <= 1e-9 * abs(r64.E0)


@pytest.mark.parametrize("a", [0, 3])
def test_column_blocked_product_and_solve(a, monkeypatch):
    """The column-blocked coded FP32 layout (built for vectors larger than L2;
    QMB_CB_SHIFT=10 forces 1024-row blocks here): the FP32 product equals the
    oracle's matrix product to FP32 rounding and the plain sliced-ELL product
    to 2e-6 relative; the FP64 values share its packed entries through an
    FP64 dictionary, and the FP64 product matches the oracle to 1e-12; mixed,
    FP64 and FP32 solves on it match the oracle's FP64 ground energy (scipy
    eigsh)."""
    import torch
    L, k = 20, 10
    perm, ch = q.translation_group(L)
    terms = q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), [1.0] * L + [0.4] * L, 0.8)
    s = q.Sector(L, k, perm).set_irrep(ch[a])
    plain = q.Hamiltonian(s, terms)
    monkeypatch.setenv("QMB_CB_SHIFT", "10")
    hb = q.Hamiltonian(s, terms)
    assert hb.info.coded == 1 and plain.info.coded == 0
    assert hb.info.n_codes >= 1
    g = oracle_group(perm, ch)
    sec = O.build_sector(g, k)
    rows = O.active_rows(sec, a)
    rc, ind, val, tr = O.ell_terms(sec, oracle_terms(terms), a, 2 * terms.n_terms + 1)
    M = O.ell_to_csr(ind, val, tr, rows)
    n = M.shape[0]
    assert n == hb.info.n_rows and n > 4 * 1024
    rng = np.random.default_rng(a)
    xh = rng.standard_normal(n) + (1j * rng.standard_normal(n) if hb.info.is_complex else 0)
    dt = torch.complex64 if hb.info.is_complex else torch.float32
    x = torch.tensor(xh, dtype=dt, device="cuda")
    y1, y2 = torch.empty_like(x), torch.empty_like(x)
    for h, y in ((hb, y1), (plain, y2)):
        q.check(q.lib().qmb_hv(h.h, q._capi.PREC_FP32, q._capi.C.c_void_p(x.data_ptr()), q._capi.C.c_void_p(y.data_ptr()), None))
    torch.cuda.synchronize()
    want = M @ x.cpu().numpy().astype(np.complex128 if hb.info.is_complex else np.float64)
    got = y1.cpu().numpy()
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 2e-6 * scale
    assert np.abs(got - y2.cpu().numpy()).max() <= 2e-6 * scale
    # the FP64 values share the packed entries through an FP64 dictionary
    assert hb.info.coded_fp64 == 1
    dt64 = torch.complex128 if hb.info.is_complex else torch.float64
    x64 = torch.tensor(xh, dtype=dt64, device="cuda")
    z1, z2 = torch.empty_like(x64), torch.empty_like(x64)
    for h, y in ((hb, z1), (plain, z2)):
        q.check(q.lib().qmb_hv(h.h, q._capi.PREC_FP64, q._capi.C.c_void_p(x64.data_ptr()), q._capi.C.c_void_p(y.data_ptr()), None))
    torch.cuda.synchronize()
    want64 = M @ xh
    assert np.abs(z1.cpu().numpy() - want64).max() <= 1e-12 * np.abs(want64).max()
    assert np.abs(z1.cpu().numpy() - z2.cpu().numpy()).max() <= 1e-12 * np.abs(want64).max()
    e = O.ground_energy_sparse(M)
    r = hb.lanczos(mode=q._capi.MODE_MIXED, tol=1e-12)
    assert abs(r.E0 - e) <= 1e-10 * abs(e), (r.E0, e)
    r64 = hb.lanczos(mode=q._capi.MODE_FP64, tol=1e-12)
    assert abs(r64.E0 - e) <= 1e-10 * abs(e), (r64.E0, e)
    r32 = hb.lanczos(mode=q._capi.MODE_FP32, tol=1e-12, allow_unconverged=True)
    assert abs(r32.E0 - e) <= 1e-5 * abs(e), (r32.E0, e)
