"""CPU tests of the C ABI: the library loads, exports every declared symbol,
and its host-side model/symmetry helpers reproduce the reference's classes
(T_standard compiled from the reference sources into oracle/_ref)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
import qmbcuda_b200 as q

A = q._capi
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "qmb_b200.h")).read()
    return sorted(set(re.findall(r"QMB_API[^;(]*?\b(qmb_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    syms = declared_symbols()
    assert len(syms) >= 39
    lib = C.CDLL(A.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) == set(A.SIGNATURES), set(syms) ^ set(A.SIGNATURES)


def test_abi_version_and_status_strings():
    assert q.lib().qmb_abi_version() == 1
    assert q.lib().qmb_status_string(A.QMB_ERR_ELL_OVERFLOW) == b"ELL row overflow"


def test_invalid_arguments_are_reported_not_thrown():
    st = q.lib().qmb_sector_create(None, None)
    assert st == A.QMB_ERR_INVALID
    assert b"null" in q.lib().qmb_last_error()
    perm = np.array([[0, 0, 1]], np.uint32)  # not a permutation
    d = A.SectorDesc(3, 1, 1, perm.ctypes.data_as(C.POINTER(C.c_uint32)), 0, 0)
    h = C.c_void_p()
    assert q.lib().qmb_sector_create(C.byref(d), C.byref(h)) == A.QMB_ERR_INVALID
    d = A.SectorDesc(5, 2, 1, np.arange(5, dtype=np.uint32).ctypes.data_as(C.POINTER(C.c_uint32)), 1, 0)
    assert q.lib().qmb_sector_create(C.byref(d), C.byref(h)) == A.QMB_ERR_INVALID  # flip needs 2n=L


def test_gpu_entry_points_fail_cleanly_without_device():
    if q.lib().qmb_device_count() > 0:
        pytest.skip("a device is visible")
    with pytest.raises(q.QMBError) as e:
        q.Sector(8, 4, np.arange(8, dtype=np.uint32)[None])
    assert e.value.status == A.QMB_ERR_NO_DEVICE


def _tstd_ours(N1, N2, M, A4, rx, ry, J, rng_, intra, inter):
    g = q.geometry(N1, N2, A4, rx, ry)
    Jc = A.cplx_buf(J)
    rg = np.ascontiguousarray(rng_, np.float64)
    cap = 20000
    ti = np.zeros(cap, np.int32); tj = np.zeros(cap, np.int32); tv = np.zeros(2 * cap); n = C.c_int()
    q.check(q.lib().qmb_tstandard_pairs(C.byref(g), len(J), A.ptr(Jc), A.ptr(rg), intra, inter, cap,
                                        A.ptr(ti), A.ptr(tj), A.ptr(tv), C.byref(n)))
    m = n.value
    return ti[:m], tj[:m], tv[: 2 * m].view(np.complex128)


def _tstd_ref(N1, N2, M, A4, rx, ry, J, rng_, intra, inter):
    R = O.ref()
    cap = 20000
    ti = np.zeros(cap, np.int32); tj = np.zeros(cap, np.int32); tv = np.zeros(2 * cap, np.float32)
    L = N1 * N2 * M
    r1 = np.zeros(L, np.float32); r2 = np.zeros(L, np.float32)
    n = R.ref_tstandard_complex(N1, N2, M, np.asarray(A4, np.float32), np.asarray(rx, np.float32),
                                np.asarray(ry, np.float32), len(J),
                                np.ascontiguousarray(np.asarray(J, np.complex64)).view(np.float32),
                                np.asarray(rng_, np.float32), intra, inter, cap, ti, tj, tv, r1, r2)
    return ti[:n], tj[:n], tv[: 2 * n].view(np.complex64), r1, r2


SQ = (1.0, 0.0, 0.0, 1.0)
TRI = (1.0, 0.5, 0.0, np.sqrt(3.0) / 2.0)
TST = [
    ("chain16", 16, 1, 1, SQ, (0.0,), (0.0,), [1.0], [1.0001], 1, 1),
    ("chain12_j2", 12, 1, 1, SQ, (0.0,), (0.0,), [1.0, 0.5], [1.0001, 2.0001], 1, 1),
    ("square6x4_open", 6, 4, 1, SQ, (0.0,), (0.0,), [1.0, 0.15], [1.0001, 1.4143], 1, 0),
    ("square2x4_pbc", 2, 4, 1, SQ, (0.0,), (0.0,), [1.0, 0.15j + 0.15], [1.0001, 1.4143], 1, 1),
    ("tri4x4_pbc", 4, 4, 1, TRI, (0.0,), (0.0,), [1.0, 0.15], [1.0001, 1.733], 1, 1),
    ("honeycomb2x2", 2, 2, 2, TRI, (0.0, 0.5), (0.0, 0.2886751), [1.0], [0.6], 1, 1),
]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("c", TST, ids=[c[0] for c in TST])
def test_tstandard_pairs_match_reference(c):
    name, *args = c
    ti, tj, tv = _tstd_ours(*args)
    rti, rtj, rtv, r1, r2 = _tstd_ref(*args)
    assert np.array_equal(ti, rti) and np.array_equal(tj, rtj)
    np.testing.assert_allclose(tv, rtv, rtol=1e-7)
    g = q.geometry(args[0], args[1], args[3], args[4], args[5])
    L = args[0] * args[1] * args[2]
    R1 = np.zeros(L); R2 = np.zeros(L)
    q.check(q.lib().qmb_geometry_sites(C.byref(g), A.ptr(R1), A.ptr(R2)))
    np.testing.assert_allclose(R1, r1, atol=1e-6)
    np.testing.assert_allclose(R2, r2, atol=1e-6)


def test_translation_group_is_an_abelian_group_with_its_characters():
    for N1, N2, M in ((10, 1, 1), (4, 3, 1), (2, 2, 2)):
        perm, ch = q.translation_group(N1, N2, M)
        G, L = perm.shape
        assert np.array_equal(perm[0], np.arange(L))
        # closure and character homomorphism: chi(g h) = chi(g) chi(h)
        for a in range(G):
            for b in range(G):
                comp = perm[b][perm[a]]  # apply a then b
                c = [i for i in range(G) if np.array_equal(perm[i], comp)]
                assert len(c) == 1
                np.testing.assert_allclose(ch[:, c[0]], ch[:, a] * ch[:, b], atol=1e-12)
        og = O.translation_group(N1, N2, M)
        assert np.array_equal(perm, og.perm)
        np.testing.assert_allclose(ch, og.chars, atol=1e-12)


def test_group_elem_arr_layout_is_the_inverse_site_map():
    # a shift by one site on a ring: site q moves to q+1, so perm[q+1] = q
    L = 6
    R1 = np.arange(L, dtype=np.float64); R2 = np.zeros(L)
    TR1 = ((R1 + 1) % L)[None, :].copy(); TR2 = np.zeros((1, L))
    perm = np.zeros((1, L), np.uint32)
    q.check(q.lib().qmb_group_elem_arr(L, 1, A.ptr(R1), A.ptr(R2), A.ptr(TR1), A.ptr(TR2), A.ptr(perm)))
    assert list(perm[0]) == [5, 0, 1, 2, 3, 4]
    TR1[0, 0] = 0.5  # no image
    assert q.lib().qmb_group_elem_arr(L, 1, A.ptr(R1), A.ptr(R2), A.ptr(TR1), A.ptr(TR2), A.ptr(perm)) == A.QMB_ERR_INVALID


def test_rotation_group_c4_on_square():
    from helpers import rotations_4x4
    perm, ch = rotations_4x4()
    assert perm.shape == (4, 16)
    assert np.array_equal(perm[0], np.arange(16))
    four = np.arange(16)
    for _ in range(4):
        four = perm[1][four]
    assert np.array_equal(four, np.arange(16))


def test_extended_xxx_shells_and_heisenberg_terms_square_2x4():
    """CreateHeisenbergXXXSquare(2, 4, {1, 0.15}) + BuildOperatorVecs shape."""
    g = q.geometry(2, 4)
    cap = 4096
    rows = np.zeros(4 * cap, np.int32); Jo = np.zeros(cap); n = C.c_int()
    Jv = np.array([1.0, 0.15])
    q.check(q.lib().qmb_extended_xxx_shells(C.byref(g), 2, A.ptr(Jv), cap, A.ptr(rows), A.ptr(Jo), C.byref(n)))
    m = n.value
    rows = rows[: 4 * m].reshape(m, 4)
    Jo = Jo[:m]
    d = np.hypot(rows[:, 0], rows[:, 1])
    assert np.all(np.diff(d) >= -1e-6)            # sorted by distance
    assert set(np.round(d, 4)) == {1.0, 1.4142}    # two shells
    assert np.all(Jo[np.isclose(d, 1.0)] == 1.0) and np.allclose(Jo[np.isclose(d, 1.4142, atol=1e-3)], 0.15)
    Jxy = A.cplx_buf(Jo[:m].astype(np.complex128))
    n_ops = np.zeros(cap, np.int32); codes = np.zeros(2 * cap, np.int32); sites = np.zeros(2 * cap, np.int32)
    sc = np.zeros(2 * cap); nt = C.c_int()
    r = np.ascontiguousarray(rows.ravel())
    q.check(q.lib().qmb_heisenberg_terms(C.byref(g), m, A.ptr(r), A.ptr(Jxy), m, A.ptr(r), A.ptr(Jo[:m].copy()),
                                         1, 1, cap, A.ptr(n_ops), A.ptr(codes), A.ptr(sites), A.ptr(sc), C.byref(nt)))
    H = nt.value
    assert H == 8 * 2 * m
    codes = codes[: 2 * H].reshape(H, 2)
    # per unit cell: m hopping terms [Sm, Sp] then m Sz Sz terms
    assert (codes[:m] == [A.OP_SM, A.OP_SP]).all() and (codes[m:2 * m] == [A.OP_SZ, A.OP_SZ]).all()
    # inter = false drops every term (Heisenberg.cu:57)
    q.check(q.lib().qmb_heisenberg_terms(C.byref(g), m, A.ptr(r), A.ptr(Jxy), m, A.ptr(r), A.ptr(Jo[:m].copy()),
                                         1, 0, cap, A.ptr(n_ops), A.ptr(codes.ravel().copy()), A.ptr(sites),
                                         A.ptr(sc), C.byref(nt)))
    assert nt.value == 0


def test_terms_from_pairs_rules():
    ti = np.array([0, 1, 2, 2], np.int32); tj = np.array([1, 0, 2, 0], np.int32)
    tv = A.cplx_buf(np.array([1.0, 1.0, 1.0, 2.0 + 1j]))
    cap = 16
    n_ops = np.zeros(cap, np.int32); codes = np.zeros(2 * cap, np.int32); sites = np.zeros(2 * cap, np.int32)
    sc = np.zeros(2 * cap); nt = C.c_int()
    q.check(q.lib().qmb_terms_from_pairs(4, A.ptr(ti), A.ptr(tj), A.ptr(tv), 0.5, 2.0, 0, cap, A.ptr(n_ops),
                                         A.ptr(codes), A.ptr(sites), A.ptr(sc), C.byref(nt)))
    assert nt.value == 7  # the self pair (2, 2) gets no hopping term
    c = codes[:14].reshape(7, 2)
    assert (c[0] == [A.OP_SZ, A.OP_SZ]).all() and (c[1] == [A.OP_SM, A.OP_SP]).all()
    s = sc[:14].view(np.complex128)
    assert s[0] == 2.0 and s[1] == 0.5 and s[6] == (2.0 + 1j) * 0.5
