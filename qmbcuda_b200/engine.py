"""Handle wrappers over the C ABI: sectors, Hamiltonians, Lanczos, batches.

Every method calls into libqmb_b200.so; arrays cross the boundary as numpy
host buffers (or raw device pointers for the device-side entry points).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _capi as A
from ._capi import check, cplx_buf, lib, ptr


@dataclass
class TermTable:
    """Operator tables in the layout of the reference's OperatorVectors:
    op codes and scalars as the GPU layer consumes them (already conjugated)."""

    n_ops: np.ndarray   # [H] int32
    codes: np.ndarray   # [H, C] int32
    sites: np.ndarray   # [H, C] int32
    scalar: np.ndarray  # [H] complex128

    def __post_init__(self):
        self.n_ops = np.ascontiguousarray(self.n_ops, np.int32)
        self.codes = np.ascontiguousarray(np.atleast_2d(self.codes), np.int32)
        self.sites = np.ascontiguousarray(np.atleast_2d(self.sites), np.int32)
        self.scalar = np.ascontiguousarray(self.scalar, np.complex128)
        self._sc = cplx_buf(self.scalar)

    @property
    def n_terms(self) -> int:
        return int(self.n_ops.shape[0])

    def c(self) -> A.Terms:
        t = A.Terms()
        t.n_terms = self.n_terms
        t.n_col = int(self.codes.shape[1]) if self.n_terms else 1
        t.n_ops = self.n_ops.ctypes.data_as(C.POINTER(C.c_int))
        t.op_code = self.codes.ctypes.data_as(C.POINTER(C.c_int))
        t.op_site = self.sites.ctypes.data_as(C.POINTER(C.c_int))
        t.scalar = self._sc.ctypes.data_as(C.POINTER(C.c_double))
        return t

    def __add__(self, other: "TermTable") -> "TermTable":
        w = max(self.codes.shape[1], other.codes.shape[1])
        pad = lambda a: np.pad(a, ((0, 0), (0, w - a.shape[1])))
        return TermTable(np.concatenate([self.n_ops, other.n_ops]),
                         np.concatenate([pad(self.codes), pad(other.codes)]),
                         np.concatenate([pad(self.sites), pad(other.sites)]),
                         np.concatenate([self.scalar, other.scalar]))


def xxz_terms(bonds, Jxy, Jz, part: str = "all") -> TermTable:
    """H = sum_b Jxy_b/2 (S+_i S-_j + S-_i S+_j) + Jz_b Sz_i Sz_j (physical
    convention) as GPU-layer tables.  part: "all", "xy" or "z"."""
    bonds = list(bonds)
    jxy = np.broadcast_to(np.asarray(Jxy, np.complex128), (len(bonds),))
    jz = np.broadcast_to(np.asarray(Jz, np.float64), (len(bonds),))
    n_ops, codes, sites, sc = [], [], [], []
    for (i, j), a, b in zip(bonds, jxy, jz):
        if part in ("all", "xy"):
            # S+_i S-_j: conjugated decode row [Sm(i), Sp(j)], scalar conj(J/2)
            for (p, q), s in (((i, j), np.conj(a) / 2), ((j, i), a / 2)):
                n_ops.append(2); codes.append([A.OP_SM, A.OP_SP]); sites.append([p, q]); sc.append(s)
        if part in ("all", "z"):
            n_ops.append(2); codes.append([A.OP_SZ, A.OP_SZ]); sites.append([i, j]); sc.append(b)
    if not n_ops:
        return TermTable(np.zeros(0, np.int32), np.zeros((0, 2), np.int32),
                         np.zeros((0, 2), np.int32), np.zeros(0))
    return TermTable(np.array(n_ops), np.array(codes), np.array(sites), np.array(sc))


_OP_CODE = {"Sz": A.OP_SZ, "Sp": A.OP_SP, "Sm": A.OP_SM, "I": A.OP_I}
_DAGGER = {A.OP_SZ: A.OP_SZ, A.OP_SP: A.OP_SM, A.OP_SM: A.OP_SP, A.OP_I: A.OP_I}


def operator_terms(terms) -> TermTable:
    """A physical operator sum_t s_t O_t1 O_t2 ... O_tk as GPU-layer tables.

    terms: iterable of (scalar, [(kind, site), ...]) with kind "Sz", "Sp",
    "Sm" or "I" (or the QMB_OP_* codes), factors in written order.  Each
    table row holds the factors daggered, in written order, and the conjugated
    product of scalars: the tables ComputeStaticExpValZeroT builds from a
    ManyBodyOperator (exact_diagonalization/
    HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:434-455)."""
    terms = list(terms)
    width = max([len(f) for _, f in terms] + [1])
    n_ops = np.zeros(len(terms), np.int32)
    codes = np.zeros((len(terms), width), np.int32)
    sites = np.zeros((len(terms), width), np.int32)
    sc = np.zeros(len(terms), np.complex128)
    for t, (s, factors) in enumerate(terms):
        n_ops[t] = len(factors)
        for j, (kind, site) in enumerate(factors):
            codes[t, j] = _DAGGER[_OP_CODE[kind] if isinstance(kind, str) else int(kind)]
            sites[t, j] = site
        sc[t] = np.conj(s)
    return TermTable(n_ops, codes, sites, sc)


def fourier_terms(kind: str, k, N1: int, N2: int, a=(1.0, 0.0, 0.0, 1.0), n_sub: int = 1, alpha: int = 0,
                  sign: int = 1):
    """Factors of the Fourier operator O_k = N^-1/2 sum_cells e^{i k.r} O(site),
    r = i a1 + j a2, site = (i N2 + j) n_sub + alpha, as FourierOperator
    (quantum_operators/ArbitraryOperator.cu:246-282); sign=-1 gives O_{-k}.
    Returns [(scalar, [(kind, site)])] for operator_terms or products."""
    a1 = np.array([a[0], a[2]])
    a2 = np.array([a[1], a[3]])
    kk = sign * np.asarray(k, np.float64)
    out = []
    for i in range(N1):
        for j in range(N2):
            r = i * a1 + j * a2
            out.append((np.exp(1j * float(kk @ r)) / np.sqrt(N1 * N2), [(kind, (i * N2 + j) * n_sub + alpha)]))
    return out


def multiply_terms(x, y):
    """Product of two operators in (scalar, factors) form (factors of x first),
    as ManyBodyOperator::operator* (ArbitraryOperator.cu:171-186)."""
    return [(sa * sb, list(fa) + list(fb)) for sa, fa in x for sb, fb in y]


def reciprocal_basis(a=(1.0, 0.0, 0.0, 1.0)):
    """The matrix of ReciprocalBasisVectors (geometry/base.cpp:7-16) for
    A_mat given row-major as a: its columns are b1, b2 with
    a_i . b_j = 2 pi delta_ij (FullFourierOperator's k uses the columns)."""
    det = a[0] * a[3] - a[1] * a[2]
    c = 2.0 * np.pi / det
    return np.array([[c * a[3], -c * a[2]], [-c * a[1], c * a[0]]])


def chain_bonds(L: int, r: int = 1):
    return [(i, (i + r) % L) for i in range(L)]


def square_bonds(N1: int, N2: int):
    out = []
    for i1 in range(N1):
        for i2 in range(N2):
            q = i1 * N2 + i2
            out.append((q, ((i1 + 1) % N1) * N2 + i2))
            out.append((q, i1 * N2 + (i2 + 1) % N2))
    return out


def geometry(N1: int, N2: int = 1, a=(1.0, 0.0, 0.0, 1.0), rx=(0.0,), ry=(0.0,)):
    g = A.Geometry()
    g.N1, g.N2, g.n_sub = N1, N2, len(rx)
    for i in range(4):
        g.a[i] = a[i]
    g._rx = np.ascontiguousarray(rx, np.float64)
    g._ry = np.ascontiguousarray(ry, np.float64)
    g.rx = g._rx.ctypes.data_as(C.POINTER(C.c_double))
    g.ry = g._ry.ctypes.data_as(C.POINTER(C.c_double))
    return g


def translation_group(N1: int, N2: int = 1, n_sub: int = 1):
    """(perm [G, L], chars [G, G] complex) of the lattice translations."""
    g = geometry(N1, N2, rx=(0.0,) * n_sub, ry=(0.0,) * n_sub)
    L, G = N1 * N2 * n_sub, N1 * N2
    perm = np.zeros((G, L), np.uint32)
    ch = np.zeros(2 * G * G)
    check(lib().qmb_group_translations(C.byref(g), ptr(perm), ptr(ch)))
    return perm, ch.view(np.complex128).reshape(G, G)


def with_spin_flip(chars_row, parity: int) -> np.ndarray:
    """Character row over e = z*G + g for spin inversion with parity +-1."""
    chars_row = np.asarray(chars_row, np.complex128)
    return np.concatenate([chars_row, parity * chars_row])


class Sector:
    """Fixed-Sz sector reduced by a group (qmb_sector)."""

    def __init__(self, L: int, n_up: int, perm, spin_flip: bool = False, device: int = 0):
        self._perm = np.ascontiguousarray(np.atleast_2d(perm), np.uint32)
        d = A.SectorDesc(L, n_up, self._perm.shape[0],
                         self._perm.ctypes.data_as(C.POINTER(C.c_uint32)), int(spin_flip), device)
        h = C.c_void_p()
        check(lib().qmb_sector_create(C.byref(d), C.byref(h)))
        self.h = h
        self.L, self.n_up = L, n_up

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Sector":
        """A sector (and its saved irrep) from a table file of save()."""
        h = C.c_void_p()
        check(lib().qmb_sector_load(os.fsencode(path), device, C.byref(h)))
        s = cls.__new__(cls)
        s.h = h
        s._perm = None
        s.L = s.n_up = None
        return s

    def save(self, path: str) -> None:
        check(lib().qmb_sector_save(self.h, os.fsencode(path)))

    def close(self):
        if getattr(self, "h", None):
            lib().qmb_sector_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_irrep(self, chars, tol_norm: float = 1e-5):
        c = cplx_buf(chars)
        check(lib().qmb_sector_set_irrep(self.h, ptr(c), tol_norm))
        return self

    @property
    def info(self) -> A.SectorInfo:
        i = A.SectorInfo()
        check(lib().qmb_sector_get_info(self.h, C.byref(i)))
        return i

    def reps(self) -> np.ndarray:
        n = self.info.n_orbits
        out = np.zeros(n, np.uint64)
        check(lib().qmb_sector_reps(self.h, ptr(out), n))
        return out

    def norms(self) -> np.ndarray:
        n = self.info.n_orbits
        out = np.zeros(n)
        check(lib().qmb_sector_norms(self.h, ptr(out), n))
        return out

    def active(self) -> np.ndarray:
        n = self.info.n_active
        out = np.zeros(max(n, 1), np.int64)
        check(lib().qmb_sector_active(self.h, ptr(out), n))
        return out[:n]

    def orbit_map(self) -> np.ndarray:
        n = 2 * self.info.n_states
        out = np.zeros(n, np.uint32)
        check(lib().qmb_sector_orbit_map(self.h, ptr(out), n))
        return out

    def lookup(self, states):
        s = np.ascontiguousarray(states, np.uint64)
        o = np.zeros(len(s), np.int64)
        e = np.zeros(len(s), np.int32)
        check(lib().qmb_sector_lookup(self.h, ptr(s), len(s), ptr(o), ptr(e)))
        return o, e


def export_ref(sector: Sector, terms: TermTable, W: int):
    R = sector.info.n_orbits
    ind = np.zeros(R * W, np.uint32)
    val = np.zeros(2 * R * W)
    track = np.zeros(R, np.int16)
    t = terms.c()
    check(lib().qmb_ham_export_ref(sector.h, C.byref(t), W, ptr(ind), ptr(val), ptr(track)))
    return ind.reshape(R, W), val.view(np.complex128).reshape(R, W), track


def export_nosym(L: int, n_up: int, terms: TermTable, W: int, device: int = 0):
    from math import comb
    n = comb(L, n_up)
    ind = np.zeros(n * W, np.uint32)
    val = np.zeros(2 * n * W)
    track = np.zeros(n, np.int16)
    t = terms.c()
    check(lib().qmb_ham_export_nosym(L, n_up, C.byref(t), W, ptr(ind), ptr(val), ptr(track), device))
    return ind.reshape(n, W), val.view(np.complex128).reshape(n, W), track


def save_ref_ell(path: str, ind, val, track) -> None:
    """Reference-layout ELL tables (host arrays) to a table file."""
    ind = np.ascontiguousarray(ind, np.uint32)
    cplx = np.iscomplexobj(val)
    val = np.ascontiguousarray(val, np.complex64 if cplx else np.float32)
    track = np.ascontiguousarray(track, np.int16)
    R, W = ind.shape
    assert val.shape == (R, W) and track.shape == (R,)
    check(lib().qmb_ref_ell_save(os.fsencode(path), R, W, ptr(ind), ptr(val), ptr(track), int(cplx)))


def load_ref_ell(path: str):
    """(ind, val, track) of a reference-layout ELL table file."""
    R, W, cp = C.c_int64(), C.c_int(), C.c_int()
    p = os.fsencode(path)
    check(lib().qmb_ref_ell_load(p, C.byref(R), C.byref(W), C.byref(cp), None, None, None, 0))
    ind = np.zeros((R.value, W.value), np.uint32)
    val = np.zeros((R.value, W.value), np.complex64 if cp.value else np.float32)
    track = np.zeros(R.value, np.int16)
    check(lib().qmb_ref_ell_load(p, C.byref(R), C.byref(W), C.byref(cp), ptr(ind), ptr(val), ptr(track),
                                 R.value))
    return ind, val, track


class Hamiltonian:
    """Matrix of a sector's irrep in sliced ELL on the device (qmb_ham)."""

    def __init__(self, sector: Sector, terms: TermTable, prec: int = A.PREC_FP64 | A.PREC_FP32):
        self.sector = sector
        self.terms = terms
        t = terms.c()
        h = C.c_void_p()
        check(lib().qmb_ham_create(sector.h, C.byref(t), prec, C.byref(h)))
        self.h = h

    @classmethod
    def load(cls, sector: Sector, path: str) -> "Hamiltonian":
        """A matrix from a table file of save(), on the sector irrep it was built for."""
        h = C.c_void_p()
        check(lib().qmb_ham_load(sector.h, os.fsencode(path), C.byref(h)))
        m = cls.__new__(cls)
        m.sector, m.terms, m.h = sector, None, h
        return m

    def save(self, path: str) -> None:
        check(lib().qmb_ham_save(self.h, os.fsencode(path)))

    def close(self):
        if getattr(self, "h", None):
            lib().qmb_ham_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def info(self) -> A.HamInfo:
        i = A.HamInfo()
        check(lib().qmb_ham_get_info(self.h, C.byref(i)))
        return i

    def dtype(self, prec: int):
        cplx = bool(self.info.is_complex)
        if prec == A.PREC_FP64:
            return np.complex128 if cplx else np.float64
        return np.complex64 if cplx else np.float32

    def hv_host(self, x, prec: int = A.PREC_FP64) -> np.ndarray:
        x = np.ascontiguousarray(x, self.dtype(prec))
        y = np.zeros_like(x)
        check(lib().qmb_hv_host(self.h, prec, ptr(x), ptr(y)))
        return y

    def hv_dev(self, x_ptr: int, y_ptr: int, prec: int = A.PREC_FP64, stream: int = 0,
               matrix_free: bool = False):
        f = lib().qmb_hv_matrix_free if matrix_free else lib().qmb_hv
        check(f(self.h, prec, C.c_void_p(x_ptr), C.c_void_p(y_ptr), C.c_void_p(stream)))

    def lanczos(self, n_coeffs: int = 0, allow_unconverged: bool = False, **kw):
        o = A.default_opts(**kw)
        r = A.LanczosResult()
        cf = np.zeros(max(n_coeffs, 1))
        st = lib().qmb_lanczos(self.h, C.byref(o), C.byref(r), ptr(cf) if n_coeffs else None,
                               n_coeffs)
        if not (allow_unconverged and st == A.QMB_ERR_NOT_CONVERGED):
            check(st)
        return (r, cf[:n_coeffs]) if n_coeffs else r

    def ground_state(self) -> np.ndarray:
        n = self.info.n_rows
        out = np.zeros(n, self.dtype(A.PREC_FP64))
        check(lib().qmb_ground_state(self.h, ptr(out), n))
        return out

    def set_ground_state(self, psi) -> None:
        psi = np.ascontiguousarray(psi, self.dtype(A.PREC_FP64))
        check(lib().qmb_set_ground_state(self.h, ptr(psi), psi.shape[0]))

    def expval(self, ops, psi_dev: int = 0) -> np.ndarray:
        """<psi|A_k|psi> / <psi|psi> for each TermTable A_k (operator_terms
        form) on the kept ground state, or on the device vector psi_dev."""
        single = isinstance(ops, TermTable)
        ops = [ops] if single else list(ops)
        arr = (A.Terms * max(len(ops), 1))()
        for k, t in enumerate(ops):
            arr[k] = t.c()
        out = np.zeros(2 * max(len(ops), 1))
        check(lib().qmb_expval(self.h, len(ops), arr, C.c_void_p(psi_dev) if psi_dev else None, ptr(out)))
        v = out[: 2 * len(ops)].view(np.complex128)
        return v[0] if single else v


class Batch:
    """Many coupling sets over many sectors (qmb_batch)."""

    def __init__(self, sectors, terms_xy: TermTable, terms_z: TermTable, n_sets: int,
                 device: int = 0):
        self.sectors = list(sectors)
        arr = (C.c_void_p * len(self.sectors))(*[s.h.value for s in self.sectors])
        self._arr = arr
        self._txy, self._tz = terms_xy.c(), terms_z.c()
        self._keep = (terms_xy, terms_z)
        d = A.BatchDesc(len(self.sectors), C.cast(arr, C.POINTER(C.c_void_p)),
                        C.pointer(self._txy), C.pointer(self._tz), n_sets, device)
        h = C.c_void_p()
        check(lib().qmb_batch_create(C.byref(d), C.byref(h)))
        self.h = h
        self.n_sets = n_sets

    def close(self):
        if getattr(self, "h", None):
            lib().qmb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def info(self) -> A.BatchInfo:
        i = A.BatchInfo()
        check(lib().qmb_batch_get_info(self.h, C.byref(i)))
        return i

    def layout(self):
        n = len(self.sectors)
        off = np.zeros(n + 1, np.int64)
        cp = np.zeros(n, np.int32)
        check(lib().qmb_batch_layout(self.h, ptr(off), ptr(cp)))
        return off, cp

    def solve(self, c_xy, c_z, allow_unconverged: bool = False, **kw):
        cx = np.ascontiguousarray(c_xy, np.float64)
        cz = np.ascontiguousarray(c_z, np.float64)
        E = np.zeros(self.n_sets * len(self.sectors))
        o = A.default_opts(**kw)
        r = A.LanczosResult()
        st = lib().qmb_batch_solve(self.h, ptr(cx), ptr(cz), C.byref(o), ptr(E), C.byref(r))
        if not (allow_unconverged and st == A.QMB_ERR_NOT_CONVERGED):
            check(st)
        return E.reshape(self.n_sets, len(self.sectors)), r

    def hv_dev(self, x_ptr: int, y_ptr: int, prec: int, stream: int = 0):
        check(lib().qmb_batch_hv(self.h, prec, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                 C.c_void_p(stream)))
