"""The oracle and the engine against committed outputs of the reference's own
code (tests/golden/reference_tables.npz, written by tests/golden/make_golden.py
from the reference compiled for the host).  These pins hold without the
reference sources.

Tolerances: integer tables bit-exact; the reference's FP32 values to FP32
rounding (2e-6 relative, 5e-6 absolute on ELL values); energies 1e-10.
Reference norms of exactly-null orbits are FP32 round-off (the reference's
documented defect), so the ELL rule is checked on the reference's own norms.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "reference_tables.npz"))

CASES = [("chain10", lambda: O.translation_group(10), 5, "chain"),
         ("square2x4", lambda: O.translation_group(2, 4), 4, "ring")]


def _bonds(kind, L):
    return O.chain_bonds(L) if kind == "chain" else [(i, (i + 1) % L) for i in range(L)]


@pytest.mark.parametrize("name,mk,k,kind", CASES, ids=[c[0] for c in CASES])
def test_oracle_tables_match_golden(name, mk, k, kind):
    g = mk()
    sec = O.build_sector(g, k)
    assert np.array_equal(G[f"{name}_reps"], [O.rank(int(s)) for s in sec.reps])
    assert np.array_equal(G[f"{name}_orbit"], sec.orbit)
    nr = G[f"{name}_norms"]
    live = (nr >= 1e-5) & (sec.norms >= 1e-5)
    np.testing.assert_allclose(nr[live], sec.norms[live], rtol=2e-6)
    diff = (nr >= 1e-5) != (sec.norms >= 1e-5)
    assert (sec.norms[diff] < 1e-7).all() and (nr[diff] < 2e-4).all()


@pytest.mark.parametrize("name,mk,k,kind", CASES, ids=[c[0] for c in CASES])
def test_oracle_ell_rule_matches_golden(name, mk, k, kind):
    g = mk()
    sec = O.build_sector(g, k)
    sec_ref = O.Sector(g, k, sec.reps, G[f"{name}_norms"].astype(np.float64), sec.orbit)
    bonds = _bonds(kind, g.L)
    t = O.xxz_terms(bonds, 1.0 + 0.3j, 0.6)
    W = 2 * len(bonds) + 1
    n_irr = g.chars.shape[0]
    for a in sorted({0, 1, n_irr // 2}):
        rc, ind, val, tr = O.ell_terms(sec_ref, t, a, W)
        assert rc >= 0
        assert np.array_equal(G[f"{name}_a{a}_track"], tr)
        assert np.array_equal(G[f"{name}_a{a}_ind"], ind)
        np.testing.assert_allclose(G[f"{name}_a{a}_val"], val, rtol=0, atol=5e-6 * max(1.0, np.abs(val).max()))


@pytest.mark.parametrize("name,N1,N2,A4,J,rg", [
    ("chain16", 16, 1, (1.0, 0.0, 0.0, 1.0), [1.0], [1.0001]),
    ("square2x4_pbc", 2, 4, (1.0, 0.0, 0.0, 1.0), [1.0, 0.15 + 0.15j], [1.0001, 1.4143])])
def test_tstandard_pairs_match_golden(name, N1, N2, A4, J, rg):
    import qmbcuda_b200 as q
    A = q._capi
    g = q.geometry(N1, N2, A4)
    Jc = A.cplx_buf(J)
    r = np.ascontiguousarray(rg, np.float64)
    cap = 4000
    ti = np.zeros(cap, np.int32); tj = np.zeros(cap, np.int32); tv = np.zeros(2 * cap); n = C.c_int()
    q.check(q.lib().qmb_tstandard_pairs(C.byref(g), len(J), A.ptr(Jc), A.ptr(r), 1, 1, cap, A.ptr(ti), A.ptr(tj),
                                        A.ptr(tv), C.byref(n)))
    m = n.value
    assert np.array_equal(ti[:m], G[f"tstd_{name}_ti"]) and np.array_equal(tj[:m], G[f"tstd_{name}_tj"])
    np.testing.assert_allclose(tv[: 2 * m].view(np.complex128), G[f"tstd_{name}_tv"], rtol=1e-7)


def test_oracle_spmv_and_energies_match_golden():
    g = O.translation_group(12)
    sec = O.build_sector(g, 6)
    t = O.xxz_terms(O.chain_bonds(12), 1.0, 1.0)
    rc, ind, val, tr = O.ell_terms(sec, t, 0, 25)
    y = O.spmv(ind, val, tr, G["hv_x"].astype(np.float64)).real
    np.testing.assert_allclose(G["hv_y"], y, atol=1e-5 * np.abs(y).max())
    for a in (0, 6):
        rows = O.active_rows(sec, a)
        rc, ind, val, tr = O.ell_terms(sec, t, a, 25)
        e = O.ground_energy_dense(O.ell_to_csr(ind, val, tr, rows))
        assert abs(e - G["e0_chain12"][a]) <= 1e-10 * abs(e)


@pytest.mark.gpu
@pytest.mark.parametrize("name,mk,k,kind", CASES, ids=[c[0] for c in CASES])
def test_engine_tables_match_golden(name, mk, k, kind):
    import qmbcuda_b200 as q
    g = mk()
    s = q.Sector(g.L, k, np.ascontiguousarray(g.perm).reshape(g.G, g.L))
    reps = s.reps()
    assert np.array_equal(G[f"{name}_reps"], [O.rank(int(v)) for v in reps])
    assert np.array_equal(G[f"{name}_orbit"], s.orbit_map())


@pytest.mark.gpu
def test_engine_energies_match_golden():
    import qmbcuda_b200 as q
    L = 12
    perm, ch = q.translation_group(L)
    terms = q.xxz_terms(q.chain_bonds(L), 1.0, 1.0)
    for a in range(L):
        e_ref = G["e0_chain12"][a]
        if not np.isfinite(e_ref):
            continue
        s = q.Sector(L, L // 2, perm).set_irrep(ch[a])
        e = q.Hamiltonian(s, terms).lanczos(tol=1e-12).E0
        assert abs(e - e_ref) <= 1e-10 * abs(e_ref), (a, e, e_ref)
