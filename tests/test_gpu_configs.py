"""The larger workloads at their full sizes, checked through size-independent
properties (no dense oracle reaches these dimensions):

  L=24 XXZ chain, Delta=0.5, k=0, spin-inversion even (56,450 rows):
      mixed FP32/FP64 and plain FP64 ground energies agree to 1e-9 relative.
  L=32 J1-J2 chain (J2=0.5), Delta=1, k=0, even (9,393,119 rows):
      stored and matrix-free H*v agree; FP32 vectors with FP64
      reorthogonalisation plus FP64 refinement reach the FP64 ground energy
      to 1e-9 relative.
  6x6 square lattice, translations + spin inversion, k=(0,0), even:
      126,056,625 orbit representatives, all active; H*v is Hermitian
      (<x, H y> = <H x, y>) and stored and matrix-free products agree.
"""
import numpy as np
import pytest

import qmbcuda_b200 as q

pytestmark = pytest.mark.gpu
A = q._capi


def _mf(h, prec, x, y):
    q.check(q.lib().qmb_hv_matrix_free(h.h, prec, A.C.c_void_p(x.data_ptr()), A.C.c_void_p(y.data_ptr()), None))


def _stored(h, prec, x, y):
    q.check(q.lib().qmb_hv(h.h, prec, A.C.c_void_p(x.data_ptr()), A.C.c_void_p(y.data_ptr()), None))


def test_l24_delta05_k0_even_mixed_matches_fp64():
    L = 24
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L), 1.0, 0.5))
    assert h.info.n_rows == 56450
    r64 = h.lanczos(mode=A.MODE_FP64, tol=1e-12)
    rmx = h.lanczos(mode=A.MODE_MIXED, tol=1e-12)
    assert abs(rmx.E0 - r64.E0) <= 1e-9 * abs(r64.E0)
    assert r64.residual < 1e-6 and rmx.residual < 1e-6
    assert rmx.E0_low != 0.0 and abs(rmx.E0_low - r64.E0) < 1e-5 * abs(r64.E0)


def test_l32_j1j2_matrix_free_and_fp32_reorth():
    import torch
    L = 32
    perm, ch = q.translation_group(L)
    s = q.Sector(L, L // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    assert s.info.n_active == 9393119
    J = [1.0] * L + [0.5] * L
    h = q.Hamiltonian(s, q.xxz_terms(q.chain_bonds(L) + q.chain_bonds(L, 2), J, J))
    n = h.info.n_rows
    assert n == 9393119
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y1, y2 = torch.empty_like(x), torch.empty_like(x)
    _stored(h, A.PREC_FP64, x, y1)
    _mf(h, A.PREC_FP64, x, y2)
    torch.cuda.synchronize()
    assert float((y1 - y2).abs().max()) <= 1e-12 * float(y1.abs().max())
    r64 = h.lanczos(mode=A.MODE_FP64, tol=1e-12, max_iter=300)
    rmx = h.lanczos(mode=A.MODE_MIXED, tol=1e-12, max_iter=300, reorth=2)
    assert abs(rmx.E0 - r64.E0) <= 1e-9 * abs(r64.E0)
    assert rmx.residual < 1e-6


def test_6x6_k0_even_sector_and_hermitian_hv(monkeypatch):
    """The 6x6 k=(0,0) even sector (126 M rows): the stored and matrix-free
    FP32 products agree and are Hermitian; the matrix-free product looks its
    rows up in the hash table (the representative table is 1 GB) and gives
    the same bits as with the bucket search (QMB_MF_HASH=0)."""
    import torch
    N = 6
    perm, ch = q.translation_group(N, N)
    s = q.Sector(N * N, N * N // 2, perm, spin_flip=True)
    assert s.info.n_orbits == 126056625
    s.set_irrep(q.with_spin_flip(ch[0], 1))
    assert s.info.n_active == 126056625
    h = q.Hamiltonian(s, q.xxz_terms(q.square_bonds(N, N), 1.0, 1.0), prec=A.PREC_FP32)
    n = h.info.n_rows
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn(n, dtype=torch.float32, device="cuda", generator=g)
    z = torch.randn(n, dtype=torch.float32, device="cuda", generator=g)
    hx, hz, hx2 = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    _stored(h, A.PREC_FP32, x, hx)
    _stored(h, A.PREC_FP32, z, hz)
    _mf(h, A.PREC_FP32, x, hx2)
    monkeypatch.setenv("QMB_MF_HASH", "0")
    hx3 = torch.empty_like(x)
    _mf(h, A.PREC_FP32, x, hx3)
    monkeypatch.delenv("QMB_MF_HASH")
    torch.cuda.synchronize()
    assert torch.equal(hx2, hx3)
    assert float((hx - hx2).abs().max()) <= 1e-4 * float(hx.abs().max())
    a = float(torch.dot(z.double(), hx.double()))
    b = float(torch.dot(hz.double(), x.double()))
    assert abs(a - b) <= 1e-5 * (abs(a) + abs(b))


def test_6x6_k0_even_ground_energy():
    """6x6 Heisenberg torus, k=(0,0), spin-inversion even: the mixed form
    (FP32 phase, FP64 restart) and 200 fixed FP32 steps (FP64 reductions).
    E0/36 against the published exact-diagonalisation value -0.678872
    (Schulz, Ziman and Poilblanc, J. Phys. I France 6, 675 (1996)), which is
    quoted to six decimals; the FP32 run agrees with the mixed one to FP32
    level."""
    N = 6
    perm, ch = q.translation_group(N, N)
    s = q.Sector(N * N, N * N // 2, perm, spin_flip=True).set_irrep(q.with_spin_flip(ch[0], 1))
    h = q.Hamiltonian(s, q.xxz_terms(q.square_bonds(N, N), 1.0, 1.0), prec=A.PREC_FP32 | A.PREC_FP64)
    rmx = h.lanczos(mode=A.MODE_MIXED, max_iter=200, tol=1e-12, refine_max_iter=200)
    assert abs(rmx.E0 / 36 - (-0.678872)) < 1e-6, rmx.E0 / 36
    assert rmx.residual < 1e-6 * abs(rmx.E0)
    r32 = h.lanczos(mode=A.MODE_FP32, max_iter=200, tol=0.0, allow_unconverged=True)
    assert r32.iters == 200
    assert abs(r32.E0 - rmx.E0) < 1e-6 * abs(rmx.E0), (r32.E0, rmx.E0)
