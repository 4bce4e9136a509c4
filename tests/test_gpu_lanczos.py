"""GPU Lanczos ground states against dense FP64 diagonalisation (oracle).

Tolerances: FP64 and mixed (FP32 + FP64 refinement) modes 1e-10 relative;
FP32 mode 1e-5 relative; the reference-layout entry point (FP32 vectors,
fixed step count, cuRAND start vector) 1e-5 relative.
"""
import numpy as np
import pytest

import oracle as O
import qmbcuda_b200 as q
from helpers import oracle_group, oracle_terms

pytestmark = pytest.mark.gpu
A = q._capi


def _dense_e0(perm, chars, flip, L, k, a, terms):
    g = oracle_group(perm, chars, flip)
    sec = O.build_sector(g, k)
    W = 2 * terms.n_terms + 1
    rc, ind, val, tr = O.ell_terms(sec, oracle_terms(terms), a, W)
    M = O.ell_to_csr(ind, val, tr, O.active_rows(sec, a))
    return O.ground_energy_dense(M)


@pytest.mark.parametrize("mode,tol", [(A.MODE_FP64, 1e-10), (A.MODE_MIXED, 1e-10), (A.MODE_FP32, 1e-5)])
@pytest.mark.parametrize("a", [0, 3, 6])
def test_chain14_translation_irreps(mode, tol, a):
    L, k = 14, 7
    perm, ch = q.translation_group(L)
    terms = q.xxz_terms(q.chain_bonds(L), 1.0, 0.5)
    e_ref = _dense_e0(perm, ch, False, L, k, a, terms)
    s = q.Sector(L, k, perm).set_irrep(ch[a])
    h = q.Hamiltonian(s, terms)
    r = h.lanczos(mode=mode, max_iter=300, tol=1e-12)
    assert abs(r.E0 - e_ref) <= tol * abs(e_ref), (r.E0, e_ref)
    if mode != A.MODE_FP32:
        assert r.residual < 1e-5


def test_spin_inversion_sectors():
    L, k = 12, 6
    perm, ch = q.translation_group(L)
    terms = q.xxz_terms(q.chain_bonds(L), 1.0, 0.5)
    chf = np.block([[ch, ch], [ch, -ch]])
    for row in (0, L // 2, L, L + L // 2):  # k=0,pi with parity +1 and -1
        e_ref = _dense_e0(perm, chf, True, L, k, row, terms)
        s = q.Sector(L, k, perm, spin_flip=True).set_irrep(chf[row])
        r = q.Hamiltonian(s, terms).lanczos(mode=A.MODE_MIXED, tol=1e-12)
        assert abs(r.E0 - e_ref) <= 1e-10 * abs(e_ref)


def test_union_of_irreps_is_the_full_sector_ground_state():
    L, k = 12, 6
    perm, ch = q.translation_group(L)
    terms = q.xxz_terms(q.chain_bonds(L), 1.0, 1.0)
    e = []
    for a in range(L):
        s = q.Sector(L, k, perm).set_irrep(ch[a])
        e.append(q.Hamiltonian(s, terms).lanczos(tol=1e-12).E0)
    full = q.Sector(L, k, np.arange(L, dtype=np.uint32)[None]).set_irrep([1.0])
    e_full = q.Hamiltonian(full, terms).lanczos(tol=1e-12).E0
    assert abs(min(e) - e_full) < 1e-10 * abs(e_full)
    assert abs(e_full - (-5.3873909174)) < 1e-9  # dense FP64 value, L=12 Heisenberg chain, Sz=0


def test_config1_l16_full_reorth_150_steps():
    """L=16 chain, J=1, Delta=1, Sz=0, no symmetry, FP64, 150 steps with full
    reorthogonalisation from a seeded uniform(-1,1) start."""
    L = 16
    s = q.Sector(L, 8, np.arange(L, dtype=np.uint32)[None]).set_irrep([1.0])
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L), 1.0, 1.0))
    assert h.info.n_rows == 12870
    r = h.lanczos(mode=A.MODE_FP64, max_iter=150, tol=0.0, reorth=2, seed=20261203)
    assert r.iters == 150
    assert abs(r.E0 - (-7.1422963606)) < 1e-9
    assert r.residual < 1e-8


def test_selective_second_reorthogonalisation_pass(monkeypatch):
    """reorth=2 runs the second Gram-Schmidt pass only when the first removed
    more than 1 - 1/sqrt(2) of the vector (Kahan-Parlett); QMB_REORTH_ALWAYS=1
    runs it every step.  Same energy and residual level either way, FP64 and
    mixed, on the 150-step L=16 solve and an L=14 momentum sector."""
    L = 16
    s = q.Sector(L, 8, np.arange(L, dtype=np.uint32)[None]).set_irrep([1.0])
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L), 1.0, 1.0))
    perm, ch = q.translation_group(14)
    s2 = q.Sector(14, 7, perm).set_irrep(ch[3])
    h2 = q.Hamiltonian(s2, q.xxz_terms(q.chain_bonds(14) + q.chain_bonds(14, 2), [1.0] * 14 + [0.4] * 14, 0.8))
    for hh, kw in ((h, dict(mode=A.MODE_FP64, max_iter=150, tol=0.0, reorth=2, seed=20261203)),
                   (h2, dict(mode=A.MODE_FP64, tol=1e-12, reorth=2)),
                   (h2, dict(mode=A.MODE_MIXED, tol=1e-12, reorth=2))):
        monkeypatch.delenv("QMB_REORTH_ALWAYS", raising=False)
        r1 = hh.lanczos(**kw)
        monkeypatch.setenv("QMB_REORTH_ALWAYS", "1")
        r2 = hh.lanczos(**kw)
        assert abs(r1.E0 - r2.E0) <= 1e-12 * abs(r2.E0), (r1.E0, r2.E0)
        assert r1.residual <= 10 * r2.residual + 1e-12 * abs(r2.E0)
    assert abs(r1.E0 - h2.lanczos(mode=A.MODE_FP64, tol=1e-12).E0) <= 1e-10 * abs(r1.E0)


def test_matrix_free_solve_matches_stored():
    L, k = 16, 8
    perm, ch = q.translation_group(L)
    chf = np.concatenate([ch[0], ch[0]])
    s = q.Sector(L, k, perm, spin_flip=True).set_irrep(chf)
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), [1.0] * L + [0.5] * L, 1.0))
    r1 = h.lanczos(mode=A.MODE_FP64, tol=1e-12)
    r2 = h.lanczos(mode=A.MODE_FP64, tol=1e-12, hv=A.HV_MATRIX_FREE)
    assert abs(r1.E0 - r2.E0) < 1e-11 * abs(r1.E0)


@pytest.mark.parametrize("mode", [A.MODE_FP64, A.MODE_MIXED])
def test_wrapping_ring_regenerates_the_basis(mode, monkeypatch):
    """A Krylov ring that may not grow (QMB_LZ_RING_MAX=4 slots) wraps and
    the Ritz vector is regenerated from the seed: the energy and the ground
    state match the solve with the whole basis stored, and the regeneration
    shows in the product count."""
    L, k = 16, 8
    perm, ch = q.translation_group(L)
    s = q.Sector(L, k, perm).set_irrep(ch[0])
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), [1.0] * L + [0.4] * L, 0.8))
    r1 = h.lanczos(mode=mode, tol=1e-12, want_vector=1)
    psi1 = h.ground_state()
    monkeypatch.setenv("QMB_LZ_RING_MAX", "4")
    h2 = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), [1.0] * L + [0.4] * L, 0.8))
    r2 = h2.lanczos(mode=mode, tol=1e-12, want_vector=1)
    psi2 = h2.ground_state()
    assert abs(r2.E0 - r1.E0) <= 1e-12 * abs(r1.E0)
    assert r2.residual < 1e-6 * abs(r1.E0)
    assert r2.n_hv > r1.n_hv
    assert abs(abs(np.vdot(psi1, psi2)) - 1.0) < 1e-10


def test_ground_state_vector_and_ritz_coefficients():
    L, k = 12, 6
    perm, ch = q.translation_group(L)
    s = q.Sector(L, k, perm).set_irrep(ch[0])
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L), 1.0, 1.0))
    r, cf = h.lanczos(n_coeffs=300, tol=1e-12, want_vector=1)
    psi = h.ground_state()
    assert abs(np.linalg.norm(psi) - 1) < 1e-8
    hp = h.hv_host(psi)
    assert np.linalg.norm(hp - r.E0 * psi) < 1e-7
    assert abs(np.linalg.norm(cf[: r.iters]) - 1) < 1e-10


def test_reference_layout_lanczos_entry_point():
    """qmb_lanczos_ref_ell on a caller-owned reference-layout ELL (FP32)."""
    import torch
    L, k = 12, 6
    perm, ch = q.translation_group(L)
    s = q.Sector(L, k, perm).set_irrep(ch[0])
    terms = q.xxz_terms(q.chain_bonds(L), 1.0, 1.0)
    W = 2 * L + 1
    ind, val, tr = q.export_ref(s, terms, W)
    R = ind.shape[0]
    dind = torch.tensor(ind.astype(np.int64).ravel(), dtype=torch.int64).to(torch.int32).cuda()
    dval = torch.tensor(val.real.astype(np.float32).ravel()).cuda()
    dtr = torch.tensor(tr.astype(np.int16)).cuda()
    E = A.C.c_float()
    res = A.C.c_float()
    kry = np.zeros(120, np.float32)
    q.check(q.lib().qmb_lanczos_ref_ell(A.C.byref(E), 120, R, W, 2212456, A.C.c_void_p(dind.data_ptr()),
                                        A.C.c_void_p(dval.data_ptr()), A.C.c_void_p(dtr.data_ptr()), 0,
                                        A.ptr(kry), 1, A.C.byref(res)))
    e_ref = -5.3873909174
    assert abs(E.value - e_ref) < 1e-5 * abs(e_ref)
    assert res.value < 1e-4
