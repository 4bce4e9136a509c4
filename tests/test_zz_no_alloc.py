"""qmb_lanczos_ref_ell_noalloc against qmb_lanczos_ref_ell.

The no-allocation entry point runs the same kernels with its work vectors and
reduction scratch in a static device array, so on the same caller-owned ELL
and seed it must give the same ground energy, Ritz coefficients and residual
as the allocating entry point: energies within 1e-6 relative (both are
rounded to FP32 on output), Ritz coefficients within 1e-5, residuals within
1e-5 relative.  Two calls in a row check that nothing left in the scratch by
one call changes the next.
"""
import ctypes as C

import numpy as np
import pytest

import qmbcuda_b200 as q

pytestmark = pytest.mark.gpu
A = q._capi


def _ref_ell(a):
    """Reference-layout ELL of the L=12 Heisenberg chain, k=6, momentum irrep a."""
    import torch
    L, k = 12, 6
    perm, ch = q.translation_group(L)
    s = q.Sector(L, k, perm).set_irrep(ch[a])
    terms = q.xxz_terms(q.chain_bonds(L), 1.0, 1.0)
    W = 2 * L + 1
    ind, val, tr = q.export_ref(s, terms, W)
    cplx = a not in (0, L // 2)
    dind = torch.tensor(ind.astype(np.int64).ravel(), dtype=torch.int64).to(torch.int32).cuda()
    if cplx:
        v = np.ascontiguousarray(val.astype(np.complex64).ravel()).view(np.float32)
    else:
        v = val.real.astype(np.float32).ravel()
    dval = torch.tensor(v).cuda()
    dtr = torch.tensor(tr.astype(np.int16)).cuda()
    torch.cuda.synchronize()
    return ind.shape[0], W, cplx, (dind, dval, dtr)


def _call(fn, n_iter, R, W, cplx, bufs, extra=()):
    dind, dval, dtr = bufs
    E = C.c_float()
    res = C.c_float()
    kry = np.zeros(n_iter, np.float32)
    st = fn(C.byref(E), n_iter, R, W, 2212456, C.c_void_p(dind.data_ptr()),
            C.c_void_p(dval.data_ptr()), C.c_void_p(dtr.data_ptr()), int(cplx), A.ptr(kry), 1,
            C.byref(res), *extra)
    return st, E.value, kry, res.value


@pytest.mark.parametrize("a", [0, 3])
def test_noalloc_matches_allocating_entry_point(a):
    n_iter = 120
    R, W, cplx, bufs = _ref_ell(a)
    L = q.lib()
    st, e_ref, k_ref, r_ref = _call(L.qmb_lanczos_ref_ell, n_iter, R, W, cplx, bufs)
    q.check(st)
    for _ in range(2):
        st, e, kr, r = _call(L.qmb_lanczos_ref_ell_noalloc, n_iter, R, W, cplx, bufs, (None,))
        q.check(st)
        assert abs(e - e_ref) <= 1e-6 * abs(e_ref), (e, e_ref)
        assert np.max(np.abs(kr - k_ref)) <= 1e-5
        assert abs(r - r_ref) <= 1e-5 * max(abs(r_ref), 1e-30) + 1e-12, (r, r_ref)
    if a == 0:
        assert abs(e - (-5.3873909174)) < 1e-5 * 5.3873909174


def test_noalloc_rejects_sizes_beyond_the_scratch():
    R, W, cplx, bufs = _ref_ell(0)
    L = q.lib()
    st, *_ = _call(L.qmb_lanczos_ref_ell_noalloc, 8, 262145, W, cplx, bufs, (None,))
    assert st == A.QMB_ERR_INVALID
    assert b"262144" in L.qmb_last_error()
    st, *_ = _call(L.qmb_lanczos_ref_ell_noalloc, 1025, R, W, cplx, bufs, (None,))
    assert st == A.QMB_ERR_INVALID
    assert b"1024" in L.qmb_last_error()


def test_noalloc_at_the_scratch_limit_complex_with_ritz_vector():
    """nobv = 262144, the largest size the static scratch takes, with complex
    values and the Ritz vector (check_eig_state = 1): the FP64 Ritz vector then
    ends exactly at the end of the scratch's vector region.  The matrix is a
    ring with random diagonal d_r and complex hopping t e^{i phi} between r and
    r + 1 (reference ELL layout: slot 0 the diagonal, then r + 1 and r - 1)."""
    import torch
    n, W = 262144, 3
    rng = np.random.default_rng(7)
    d = rng.uniform(-1.0, 1.0, n)
    hop = 0.8 * np.exp(1j * 0.3)
    r = np.arange(n)
    ind = np.stack([r, (r + 1) % n, (r - 1) % n], axis=1).astype(np.uint32)
    val = np.stack([d.astype(np.complex128), np.full(n, hop), np.full(n, np.conj(hop))], axis=1)
    tr = np.full(n, W, np.int16)
    dind = torch.tensor(ind.astype(np.int64).ravel()).to(torch.int32).cuda()
    dval = torch.tensor(np.ascontiguousarray(val.astype(np.complex64).ravel()).view(np.float32)).cuda()
    dtr = torch.tensor(tr).cuda()
    torch.cuda.synchronize()
    bufs = (dind, dval, dtr)
    n_iter = 60
    L = q.lib()
    st, e_ref, k_ref, r_ref = _call(L.qmb_lanczos_ref_ell, n_iter, n, W, True, bufs)
    q.check(st)
    for _ in range(2):
        st, e, kr, res = _call(L.qmb_lanczos_ref_ell_noalloc, n_iter, n, W, True, bufs, (None,))
        q.check(st)
        assert abs(e - e_ref) <= 1e-6 * abs(e_ref), (e, e_ref)
        assert np.max(np.abs(kr - k_ref)) <= 1e-5
        assert abs(res - r_ref) <= 1e-5 * max(abs(r_ref), 1e-30) + 1e-12, (res, r_ref)
