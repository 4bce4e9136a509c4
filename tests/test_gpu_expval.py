"""Ground-state expectation values on the GPU (qmb_expval) and the seeded
eigenvector of the reference-layout path (qmb_eigvec_from_seed_ref).

Checks, with their tolerances:
  - on a given FP64 state the kernel equals the oracle's rule and the dense
    physical value to 1e-12;
  - after qmb_lanczos (FP64, tight tolerance) it equals the dense value to
    1e-7 (the state's own accuracy);
  - for products of Sz it equals the reference kernel's outputs (golden
    fixtures, FP32) to 5e-6;
  - many operators in one call (several shared-memory chunks) equal one call
    per operator to 1e-13.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O
import qmbcuda_b200 as q

pytestmark = pytest.mark.gpu
A = q._capi
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as MG  # noqa: E402

G = np.load(os.path.join(HERE, "golden", "reference_tables.npz"))


def _heis_factors(L, jz=1.0, bonds=None):
    bonds = O.chain_bonds(L) if bonds is None else bonds
    out = []
    for i, j in bonds:
        out += [(0.5, [(1, i), (2, j)]), (0.5, [(2, i), (1, j)]), (jz, [(0, i), (0, j)])]
    return out


def _engine(g, k, factors, a):
    s = q.Sector(g.L, k, np.ascontiguousarray(g.perm), spin_flip=g.flip).set_irrep(g.chars[a])
    h = q.Hamiltonian(s, q.operator_terms(factors))
    return s, h


def _oracle_state(g, k, factors, a):
    sec = O.build_sector(g, k)
    tab = O.table_from_factors(factors)
    rows = O.active_rows(sec, a)
    rc, ind, val, tr = O.ell_terms(sec, tab, a, 4 * tab.H + 1)
    M = O.ell_to_csr(ind, val, tr, rows)
    M = M.toarray() if hasattr(M, "toarray") else np.asarray(M)
    w, V = np.linalg.eigh(M)
    return sec, w[0], V[:, 0]


def _phys(g, k, factors, a, ops):
    Hd = O.dense_operator(g.L, k, O.table_from_factors(factors))
    E, psi, gap = O.irrep_ground_state(Hd, O.irrep_basis(g, a, k))
    return E, gap, [psi.conj() @ O.dense_operator(g.L, k, O.table_from_factors(x)) @ psi for x in ops]


OPS = list(MG.EV_OPS.values()) + [
    [(2.5 - 1j, [(9, 3)])],                       # identity: the scalar itself
    [(1.0, [(1, 0)])],                            # S+ changes Sz: zero
    [(0.3j, [(0, 1), (1, 2), (2, 5)]), (1.0, [(2, 4), (1, 4), (0, 4)])],
]


@pytest.mark.parametrize("a", MG.EV_IRREPS)
def test_expval_on_given_state(a):
    g = O.translation_group(10)
    f = _heis_factors(10)
    sec, e, phi = _oracle_state(g, 5, f, a)
    s, h = _engine(g, 5, f, a)
    h.set_ground_state(phi if h.info.is_complex else phi.real)
    got = h.expval([q.operator_terms(x) for x in OPS])
    E, gap, phys = _phys(g, 5, f, a, OPS)
    for x, v, p in zip(OPS, got, phys):
        assert abs(v - O.expval_sym_rule(sec, x, a, phi)) <= 1e-12, x
        assert abs(v - p) <= 1e-12, (x, v, p)
    assert abs(got[len(MG.EV_OPS)] - (2.5 - 1j)) <= 1e-13
    assert abs(got[len(MG.EV_OPS) + 1]) == 0.0


@pytest.mark.parametrize("a", MG.EV_IRREPS)
def test_expval_matches_reference_for_sz_products(a):
    g = O.translation_group(10)
    f = _heis_factors(10)
    s, h = _engine(g, 5, f, a)
    h.lanczos(mode=A.MODE_FP64, max_iter=300, tol=1e-14, want_vector=1, allow_unconverged=True)
    names = ("SzSz03", "SzSz01i", "Sz2", "SzSzSzSz")
    got = h.expval([q.operator_terms(MG.EV_OPS[n]) for n in names])
    for n, v in zip(names, got):
        assert abs(v - complex(G[f"ev_chain10_a{a}_{n}"])) <= 5e-6, (n, v)


def test_expval_after_lanczos_spin_flip_group():
    L = 12
    g = O.translation_group(L, flip=True)
    f = _heis_factors(L, 0.7, O.chain_bonds(L) + O.chain_bonds(L, 2))
    ops = [[(1.0, [(0, 0), (0, j)])] for j in range(1, 7)] + [[(1.0, [(1, 0), (2, 3)])],
                                                             [(0.5, [(1, 1), (2, 2)]), (0.5, [(2, 1), (1, 2)])]]
    for a in (0, L, L // 2, L + L // 2):
        s, h = _engine(g, L // 2, f, a)
        r = h.lanczos(mode=A.MODE_FP64, max_iter=400, tol=1e-14, want_vector=1, allow_unconverged=True)
        E, gap, phys = _phys(g, L // 2, f, a, ops)
        assert abs(r.E0 - E) <= 1e-11 * abs(E)
        got = h.expval([q.operator_terms(x) for x in ops])
        tol = max(1e-9, 20 * r.residual / max(gap, 1e-3))
        for x, v, p in zip(ops, got, phys):
            assert abs(v - p) <= tol, (a, x, v, p, r.residual)


def test_expval_complex_hamiltonian_all_irreps():
    L, k = 8, 4
    g = O.translation_group(L)
    f = []
    for i in range(L):
        j, m = (i + 1) % L, (i + 2) % L
        f += [(0.5 * np.exp(1.1j), [(1, i), (2, j)]), (0.5 * np.exp(-1.1j), [(2, i), (1, j)]), (0.8, [(0, i), (0, j)]),
              (0.6 * np.exp(0.9j), [(1, i), (2, j), (0, m)]), (0.6 * np.exp(-0.9j), [(0, m), (1, j), (2, i)])]
    ops = [[(1.0, [(1, 0), (2, 1)])], [(1.0, [(1, 0), (2, 2)])], [(1.0 + 0.5j, [(0, 0), (0, 3)])]]
    for a in range(L):
        sec, e, phi = _oracle_state(g, k, f, a)
        s, h = _engine(g, k, f, a)
        h.set_ground_state(phi)
        got = h.expval([q.operator_terms(x) for x in ops])
        E, gap, phys = _phys(g, k, f, a, ops)
        for x, v, p in zip(ops, got, phys):
            assert abs(v - p) <= 1e-12, (a, x, v, p)


def test_structure_factor_fourier_vs_real_space():
    """<Sz_q Sz_-q> from Fourier operators (all q in one call) equals the
    Fourier sum of the real-space correlators <Sz_0 Sz_j>, as the reference's
    square_brute_force_example compares its two methods."""
    L = 14
    g = O.translation_group(L)
    f = _heis_factors(L)
    s, h = _engine(g, L // 2, f, 0)
    h.lanczos(mode=A.MODE_FP64, max_iter=400, tol=1e-14, want_vector=1, allow_unconverged=True)
    b = q.reciprocal_basis((1.0, 0.0, 0.0, 1.0))
    sq = []
    for n in range(L):
        kv = n * b[:, 0] / L
        pos = q.fourier_terms("Sz", kv, L, 1)
        neg = q.fourier_terms("Sz", kv, L, 1, sign=-1)
        sq.append(q.operator_terms(q.multiply_terms(pos, neg)))
    s_fourier = h.expval(sq)
    corr = h.expval([q.operator_terms([(1.0, [("Sz", 0), ("Sz", j)])]) for j in range(L)])
    s_real = np.array([np.sum(corr * np.exp(1j * 2 * np.pi * n * np.arange(L) / L)) for n in range(L)])
    assert np.max(np.abs(s_fourier - s_real)) <= 1e-10
    assert abs(corr[0] - 0.25) <= 1e-12
    assert abs(np.sum(corr)) <= 1e-10  # total Sz = 0


def test_many_operators_span_chunks():
    """Twenty Fourier operators of an L=20 chain average to about 4200 terms,
    more than one shared-memory chunk; one call equals twenty calls."""
    L = 20
    g = O.translation_group(L)
    s, h = _engine(g, L // 2, _heis_factors(L), 0)
    h.lanczos(mode=A.MODE_FP64, max_iter=300, tol=1e-12, want_vector=1, allow_unconverged=True)
    b = q.reciprocal_basis((1.0, 0.0, 0.0, 1.0))
    ops = []
    for n in range(L):
        kv = n * b[:, 0] / L
        ops.append(q.operator_terms(q.multiply_terms(q.fourier_terms("Sz", kv, L, 1),
                                                     q.fourier_terms("Sz", kv, L, 1, sign=-1))))
    together = h.expval(ops)
    for o, v in zip(ops, together):
        assert abs(h.expval(o) - v) <= 1e-13
    assert abs(together.imag).max() <= 1e-12
    assert abs(np.mean(together.real) - 0.25) <= 1e-10  # sum_q S(q) = L <Sz_0 Sz_0>


def test_expval_errors():
    g = O.translation_group(8)
    f = _heis_factors(8)
    s, h = _engine(g, 4, f, 0)
    with pytest.raises(q.QMBError):  # no state kept yet
        h.expval(q.operator_terms([(1.0, [("Sz", 0)])]))
    h.lanczos(mode=A.MODE_FP64, want_vector=1)
    bad = q.operator_terms([(1.0, [("Sz", 0)])])
    bad.codes[0, 0] = 3  # a fermion code
    with pytest.raises(q.QMBError) as e:
        h.expval(bad)
    assert e.value.status == A.QMB_ERR_INVALID
    s.set_irrep(g.chars[1])  # the handle now describes a stale irrep
    with pytest.raises(q.QMBError):
        h.expval(q.operator_terms([(1.0, [("Sz", 0), ("Sz", 1)])]))


def test_eigvec_from_seed_ref():
    """LanczosEigenStateFromSeed replacement: the regenerated vector of a
    120-step qmb_lanczos_ref_ell solve has that solve's residual and energy."""
    import torch
    L, k = 12, 6
    g = O.translation_group(L)
    sec = O.build_sector(g, k)
    t = O.xxz_terms(O.chain_bonds(L), 1.0, 1.0)
    W = 2 * L + 1
    rc, ind, val, tr = O.ell_terms(sec, t, 0, W)
    R = sec.R
    dind = torch.tensor(ind.astype(np.int64).ravel()).to(torch.int32).cuda()
    dval = torch.tensor(val.real.astype(np.float32).ravel()).cuda()
    dtr = torch.tensor(tr.astype(np.int16)).cuda()
    E = A.C.c_float()
    res = A.C.c_float()
    n_iter = 120
    kry = np.zeros(n_iter, np.float32)
    vp = lambda x: A.C.c_void_p(x.data_ptr())
    q.check(q.lib().qmb_lanczos_ref_ell(A.C.byref(E), n_iter, R, W, 2212456, vp(dind), vp(dval), vp(dtr), 0,
                                        A.ptr(kry), 1, A.C.byref(res)))
    psi = torch.zeros(R, dtype=torch.float32, device="cuda")
    q.check(q.lib().qmb_eigvec_from_seed_ref(2212456, vp(psi), A.ptr(kry), n_iter, R, W, vp(dind), vp(dval),
                                             vp(dtr), 0))
    x = psi.cpu().numpy().astype(np.float64)
    Hx = O.spmv(ind, val, tr, x).real
    rq = float(x @ Hx / (x @ x))
    r_ref = float(np.linalg.norm(Hx - E.value * x) / R)
    assert abs(rq - E.value) <= 1e-5 * abs(E.value)
    # both residuals sit at the FP32 rounding floor here; the FP32 copy may
    # differ from the solve's FP64-accumulated vector by that floor
    assert r_ref <= max(10 * res.value, 1e-7), (r_ref, res.value)
    # 120 FP32 steps without reorthogonalisation on ~80 orbits repeat the
    # ground state (ghost copies), so sum_j c_j v_j is not of unit length --
    # as in the reference, which does not normalise either; the direction is
    # the ground state's
    M = O.ell_to_csr(ind, val, tr)
    M = M.toarray() if hasattr(M, "toarray") else np.asarray(M)
    w, V = np.linalg.eigh(M.real)
    assert 1.0 - abs(V[:, 0] @ x) / np.linalg.norm(x) <= 1e-6
