"""Oracle for the XXZ Lanczos ground-state path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's reference / cpu_baseline
legs import this module, and only as the checker.  It wraps

* ``libqmb_oracle.so``: the FP64 CPU restatement in ``qmb_oracle.c``;
* ``_ref/libqmb_ref.so``: the reference's own kernels and model classes built
  for the host from the unmodified sources (``oracle/Makefile``), used to pin
  the restatement (bit-exact tables, FP32-level values).

Group conventions follow the reference: an element is a site map ``perm`` with
``perm[q]`` = destination of the bit at site q, which is the inverse site
permutation produced by ``SymmetryClass::GetGroupElemArr``
(symmetries/SymmetryClass.cu:26-71 with utils/misc_funcs.cu:80-90); elements
of ``Tnm_group`` are ordered g = nx*N2 + ny (symmetries/Groups.cu:66-73) and
its character table is chi[a][g] = exp(2 pi i (ax*gx/N1 + ay*gy/N2)) with
a = ax*N2 + ay (symmetries/Groups.cu:75-112).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE = os.path.join(HERE, "libqmb_oracle.so")
_REF = os.path.join(HERE, "_ref", "libqmb_ref.so")

_lib = None
_ref = None

P = np.ctypeslib.ndpointer
u64p = P(np.uint64, flags="C_CONTIGUOUS")
u32p = P(np.uint32, flags="C_CONTIGUOUS")
i32p = P(np.int32, flags="C_CONTIGUOUS")
i16p = P(np.int16, flags="C_CONTIGUOUS")
f64p = P(np.float64, flags="C_CONTIGUOUS")
f32p = P(np.float32, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile the oracle (and, where the reference sources exist, _ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE):
            build()
        L = C.CDLL(_ORACLE)
        L.oc_binom.restype = C.c_uint64
        L.oc_binom.argtypes = [C.c_int, C.c_int]
        L.oc_rank.restype = C.c_uint64
        L.oc_rank.argtypes = [C.c_uint64]
        L.oc_unrank.restype = C.c_uint64
        L.oc_unrank.argtypes = [C.c_uint64, C.c_int, C.c_int]
        L.oc_enumerate.restype = C.c_int64
        L.oc_enumerate.argtypes = [C.c_int, C.c_int, u64p, C.c_int64]
        L.oc_apply.restype = C.c_uint64
        L.oc_apply.argtypes = [C.c_uint64, C.c_int, u32p, C.c_int]
        L.oc_reps.restype = C.c_int64
        L.oc_reps.argtypes = [C.c_int, C.c_int, C.c_int, u32p, C.c_int, u64p, C.c_int64]
        L.oc_norms.restype = None
        L.oc_norms.argtypes = [C.c_int, C.c_int, u32p, C.c_int, C.c_int64, u64p, C.c_int, f64p, f64p]
        L.oc_orbit_map.restype = None
        L.oc_orbit_map.argtypes = [C.c_int, C.c_int, u32p, C.c_int, C.c_int64, u64p, u32p]
        L.oc_ell_terms.restype = C.c_int
        L.oc_ell_terms.argtypes = [C.c_int, C.c_int, u32p, C.c_int, C.c_int64, u64p, u32p, f64p,
                                   C.c_int, C.c_int, f64p, C.c_double, C.c_int, C.c_int, i32p,
                                   i32p, i32p, f64p, C.c_int, u32p, f64p, i16p]
        L.oc_ell_bonds.restype = C.c_int
        L.oc_ell_bonds.argtypes = [C.c_int, C.c_int, u32p, C.c_int, C.c_int64, u64p, u32p, f64p,
                                   C.c_int, C.c_int, f64p, C.c_double, C.c_int, i32p, i32p, f64p,
                                   C.c_double, C.c_double, C.c_int, u32p, f64p, i16p]
        L.oc_ell_nosym.restype = C.c_int
        L.oc_ell_nosym.argtypes = [C.c_int, C.c_int, C.c_int, i32p, i32p, f64p, C.c_double,
                                   C.c_double, C.c_int, u32p, f64p, i16p]
        L.oc_spmv.restype = None
        L.oc_spmv.argtypes = [C.c_int64, C.c_int, u32p, f64p, i16p, f64p, f64p]
        L.oc_start_vector.restype = None
        L.oc_start_vector.argtypes = [C.c_uint64, C.c_int64, f64p]
        L.oc_expval_ref.restype = None
        L.oc_expval_ref.argtypes = [C.c_int, C.c_int, u32p, C.c_int, C.c_int64, u64p, u32p, f64p,
                                    C.c_int, C.c_int, f64p, C.c_double, C.c_int, C.c_int, i32p,
                                    i32p, i32p, f64p, f64p, C.c_int, f64p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    """The reference's kernels compiled for the host (oracle/_ref)."""
    global _ref
    if _ref is None:
        if not os.path.exists(_REF):
            raise RuntimeError("oracle/_ref/libqmb_ref.so is not built (needs the reference sources)")
        R = C.CDLL(_REF)
        R.ref_rank.restype = C.c_int
        R.ref_rank.argtypes = [C.c_uint32, C.c_int]
        R.ref_nchoosek_dev.restype = C.c_double
        R.ref_nchoosek_dev.argtypes = [C.c_double, C.c_double]
        for nm in ("ref_build_srs_real", "ref_build_srs_complex"):
            f = getattr(R, nm)
            f.restype = C.c_int
            f.argtypes = [C.c_int, C.c_int, C.c_int, u32p, C.c_int, f32p, u32p, C.c_int, u32p,
                          f32p, u32p]
        for nm in ("ref_ham_bonds_real", "ref_ham_bonds_complex"):
            f = getattr(R, nm)
            f.restype = None
            f.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, u32p, u32p,
                          C.c_int, f32p, C.c_int, f32p, C.c_float, C.c_int, i32p, i32p, f32p,
                          C.c_int, u32p, f32p, i16p]
        for nm in ("ref_ham_terms_real", "ref_ham_terms_complex"):
            f = getattr(R, nm)
            f.restype = None
            f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u32p, u32p, C.c_int, f32p, C.c_int,
                          f32p, C.c_float, C.c_int, C.c_int, i32p, i32p, i32p, f32p, C.c_int,
                          u32p, f32p, i16p]
        R.ref_ham_nosym.restype = None
        R.ref_ham_nosym.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, i32p, i32p,
                                    f32p, C.c_int, u32p, f32p, i16p]
        R.ref_spmv_host.restype = None
        R.ref_spmv_host.argtypes = [u32p, f32p, i16p, f32p, f32p, C.c_int, C.c_int, C.c_int]
        R.ref_spmv_host_sweep.restype = None
        R.ref_spmv_host_sweep.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, i32p, i32p, C.c_int]
        R.ref_spmv_kernel_complex.restype = None
        R.ref_spmv_kernel_complex.argtypes = [u32p, f32p, i16p, f32p, f32p, C.c_int, C.c_int]
        R.ref_init_random_vec.restype = None
        R.ref_init_random_vec.argtypes = [C.c_longlong, C.c_int, f32p]
        for nm in ("ref_expval_real", "ref_expval_complex"):
            f = getattr(R, nm)
            f.restype = None
            f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u32p, u32p, C.c_int, f32p, C.c_int,
                          f32p, C.c_float, C.c_int, C.c_int, i32p, i32p, i32p, f32p, f32p, f32p]
        for nm in ("ref_tstandard_real", "ref_tstandard_complex"):
            f = getattr(R, nm)
            f.restype = C.c_int
            f.argtypes = [C.c_int, C.c_int, C.c_int, f32p, f32p, f32p, C.c_int, f32p, f32p,
                          C.c_int, C.c_int, C.c_int, i32p, i32p, f32p, f32p, f32p]
        _ref = R
    return _ref


# --------------------------------------------------------------- basic maps
def binom(n: int, k: int) -> int:
    return int(lib().oc_binom(n, k))


def rank(s: int) -> int:
    return int(lib().oc_rank(s))


def unrank(r: int, L: int, k: int) -> int:
    return int(lib().oc_unrank(r, L, k))


def enumerate_sector(L: int, k: int) -> np.ndarray:
    n = binom(L, k)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    got = lib().oc_enumerate(L, k, out, n)
    assert got == n
    return out[:n]


# ------------------------------------------------------------------ groups
@dataclass
class Group:
    """Site permutations (reference layout) + optional spin inversion.

    ``perm`` is [G][L] uint32; ``chars`` is [n_irr][n_ext] complex where
    n_ext = G (no inversion) or 2G, element e = z*G + g.
    """

    L: int
    perm: np.ndarray
    chars: np.ndarray
    flip: bool = False

    @property
    def G(self) -> int:
        return self.perm.shape[0]

    @property
    def n_ext(self) -> int:
        return self.G * (2 if self.flip else 1)


def trivial_group(L: int) -> Group:
    perm = np.arange(L, dtype=np.uint32)[None, :].copy()
    return Group(L, perm, np.ones((1, 1), dtype=np.complex128))


def translation_group(N1: int, N2: int = 1, M: int = 1, flip: bool = False) -> Group:
    """Tnm_group on an N1 x N2 torus with M sublattices.

    Site q = (i1*N2 + i2)*M + a (lattice_models/ArbitrarySpinLattice.cu:43-59).
    Element g = nx*N2 + ny translates by nx*a1 + ny*a2; its reference-layout
    array is the inverse site map: bit q moves to the site at (i1-nx, i2-ny).
    With ``flip`` each element also appears composed with spin inversion and
    the character table becomes chi(g) * p^z for parity rows p = +1 then -1.
    """
    L = N1 * N2 * M
    G = N1 * N2
    perm = np.zeros((G, L), dtype=np.uint32)
    for nx in range(N1):
        for ny in range(N2):
            g = nx * N2 + ny
            for i1 in range(N1):
                for i2 in range(N2):
                    for a in range(M):
                        q = (i1 * N2 + i2) * M + a
                        dst = (((i1 - nx) % N1) * N2 + (i2 - ny) % N2) * M + a
                        perm[g, q] = dst
    ch = np.zeros((G, G), dtype=np.complex128)
    for ax in range(N1):
        for ay in range(N2):
            for gx in range(N1):
                for gy in range(N2):
                    ch[ax * N2 + ay, gx * N2 + gy] = np.exp(
                        2j * np.pi * (ax * gx / N1 + ay * gy / N2))
    if flip:
        ch = np.block([[ch, ch], [ch, -ch]])
    return Group(L, perm, ch, flip)


# ------------------------------------------------------------ sector tables
@dataclass
class Sector:
    group: Group
    k: int
    reps: np.ndarray
    norms: np.ndarray  # [R][n_irr]
    orbit: np.ndarray  # [2*C(L,k)]
    extra: dict = field(default_factory=dict)

    @property
    def R(self) -> int:
        return len(self.reps)


def build_sector(group: Group, k: int, tol_norm: float = 1e-5) -> Sector:
    L, G, ne = group.L, group.G, group.n_ext
    n = binom(L, k)
    buf = np.zeros(max(n, 1), dtype=np.uint64)
    R = lib().oc_reps(L, k, G, group.perm, ne, buf, n)
    assert R >= 0
    reps = buf[:R].copy()
    n_irr = group.chars.shape[0]
    chars = np.ascontiguousarray(group.chars.astype(np.complex128)).view(np.float64).ravel()
    norms = np.zeros(max(R * n_irr, 1))
    lib().oc_norms(L, G, group.perm, ne, R, reps, n_irr, chars, norms)
    orbit = np.zeros(max(2 * n, 1), dtype=np.uint32)
    lib().oc_orbit_map(L, G, group.perm, ne, R, reps, orbit)
    return Sector(group, k, reps, norms[: R * n_irr].reshape(R, n_irr), orbit[: 2 * n])


@dataclass
class Terms:
    """Decoded operator tables in the layout of BuildOperatorVecs
    (exact_diagonalization/HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:306-336):
    op codes already conjugated (0 Sz, 1 Sp, 2 Sm), scalars already conjugated."""

    n_ops: np.ndarray   # [H] int32
    codes: np.ndarray   # [H*C] int32
    sites: np.ndarray   # [H*C] int32
    scalar: np.ndarray  # [H] complex128
    n_col: int

    @property
    def H(self) -> int:
        return len(self.n_ops)


def xxz_terms(bonds, Jxy, Jz) -> Terms:
    """H = sum_b Jxy_b/2 (S+_i S-_j + S-_i S+_j) + Jz_b Sz_i Sz_j in table form.

    For a term S+_i S-_j (raise i, lower j) the conjugated decode row is
    [Sm(i), Sp(j)]: applied in order it lowers i then raises j."""
    n_ops, codes, sites, sc = [], [], [], []
    for (i, j), jxy, jz in zip(bonds, np.broadcast_to(Jxy, len(bonds)), np.broadcast_to(Jz, len(bonds))):
        for (a, b) in ((i, j), (j, i)):
            n_ops.append(2)
            codes += [2, 1]
            sites += [a, b]
            sc.append(np.conj(0.5 * jxy))
        n_ops.append(2)
        codes += [0, 0]
        sites += [i, j]
        sc.append(jz)
    return Terms(np.array(n_ops, np.int32), np.array(codes, np.int32), np.array(sites, np.int32),
                 np.array(sc, np.complex128), 2)


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


def ell_terms(sec: Sector, terms: Terms, alpha: int, W: int, tol_norm: float = 1e-5):
    g = sec.group
    R = sec.R
    ind = np.zeros(R * W, np.uint32)
    val = np.zeros(2 * R * W)
    track = np.zeros(R, np.int16)
    chars = np.ascontiguousarray(g.chars.astype(np.complex128)).view(np.float64).ravel()
    scal = np.ascontiguousarray(terms.scalar.astype(np.complex128)).view(np.float64).ravel()
    rc = lib().oc_ell_terms(g.L, g.G, g.perm, g.n_ext, R, sec.reps, sec.orbit,
                            np.ascontiguousarray(sec.norms.ravel()), sec.norms.shape[1], alpha,
                            chars, tol_norm, terms.H, terms.n_col, terms.n_ops, terms.codes,
                            terms.sites, scal, W, ind, val, track)
    return rc, ind.reshape(R, W), val.view(np.complex128).reshape(R, W), track


def ell_bonds(sec: Sector, ti, tj, tval, jxy_w: float, jz_w: float, alpha: int, W: int,
              tol_norm: float = 1e-5):
    g = sec.group
    R = sec.R
    ind = np.zeros(R * W, np.uint32)
    val = np.zeros(2 * R * W)
    track = np.zeros(R, np.int16)
    chars = np.ascontiguousarray(g.chars.astype(np.complex128)).view(np.float64).ravel()
    tv = np.ascontiguousarray(np.asarray(tval, np.complex128)).view(np.float64).ravel()
    rc = lib().oc_ell_bonds(g.L, g.G, g.perm, g.n_ext, R, sec.reps, sec.orbit,
                            np.ascontiguousarray(sec.norms.ravel()), sec.norms.shape[1], alpha,
                            chars, tol_norm, len(ti), np.asarray(ti, np.int32),
                            np.asarray(tj, np.int32), tv, jxy_w, jz_w, W, ind, val, track)
    return rc, ind.reshape(R, W), val.view(np.complex128).reshape(R, W), track


def ell_nosym(L: int, k: int, ti, tj, tval, jxy_w: float, jz_w: float, W: int):
    n = binom(L, k)
    ind = np.zeros(n * W, np.uint32)
    val = np.zeros(2 * n * W)
    track = np.zeros(n, np.int16)
    tv = np.ascontiguousarray(np.asarray(tval, np.complex128)).view(np.float64).ravel()
    rc = lib().oc_ell_nosym(L, k, len(ti), np.asarray(ti, np.int32), np.asarray(tj, np.int32), tv,
                            jxy_w, jz_w, W, ind, val, track)
    return rc, ind.reshape(n, W), val.view(np.complex128).reshape(n, W), track


def active_rows(sec: Sector, alpha: int, tol_norm: float = 1e-5) -> np.ndarray:
    return np.nonzero(sec.norms[:, alpha] >= tol_norm)[0]


def ell_to_csr(ind, val, track, rows=None):
    """Reference-layout ELL -> scipy CSR restricted to ``rows`` (renumbered)."""
    import scipy.sparse as sp
    R, W = ind.shape
    if rows is None:
        rows = np.arange(R)
    remap = -np.ones(R, np.int64)
    remap[rows] = np.arange(len(rows))
    r_idx, c_idx, v = [], [], []
    tr = track.astype(np.int64)
    for slot in range(W):
        sel = rows[tr[rows] > slot]
        r_idx.append(remap[sel])
        c_idx.append(remap[ind[sel, slot].astype(np.int64)])
        v.append(val[sel, slot])
    r_idx = np.concatenate(r_idx)
    c_idx = np.concatenate(c_idx)
    v = np.concatenate(v)
    assert (c_idx >= 0).all(), "an entry points at a row outside the active set"
    n = len(rows)
    return sp.csr_matrix((v, (r_idx, c_idx)), shape=(n, n))


def spmv(ind, val, track, x):
    R, W = ind.shape
    xv = np.ascontiguousarray(np.asarray(x, np.complex128)).view(np.float64).ravel()
    y = np.zeros(2 * R)
    lib().oc_spmv(R, W, np.ascontiguousarray(ind.ravel()),
                  np.ascontiguousarray(val.astype(np.complex128)).view(np.float64).ravel(),
                  track, xv, y)
    return y.view(np.complex128)


def start_vector(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().oc_start_vector(seed, n, out)
    return out


# ---------------------------------------------------------------- eigen
def ground_energy_dense(A) -> float:
    d = A.toarray() if hasattr(A, "toarray") else np.asarray(A)
    d = 0.5 * (d + d.conj().T)
    return float(np.linalg.eigvalsh(d)[0])


def lanczos_fp64(matvec, v0, n_iter: int, reorth: bool = True):
    """FP64 Lanczos with optional full reorthogonalization (two classical
    Gram-Schmidt passes); returns (E0, alphas, betas)."""
    v = np.asarray(v0, np.complex128)
    v = v / np.linalg.norm(v)
    V = [v]
    a, b = [], []
    w_prev = None
    beta = 0.0
    for j in range(n_iter):
        w = matvec(V[-1])
        if w_prev is not None:
            w = w - beta * V[-2]
        al = np.vdot(V[-1], w).real
        w = w - al * V[-1]
        if reorth:
            Vm = np.array(V)
            for _ in range(2):
                w = w - Vm.T @ (Vm.conj() @ w)
        a.append(al)
        beta = np.linalg.norm(w)
        if beta < 1e-14 or j == n_iter - 1:
            break
        b.append(beta)
        w_prev = w
        V.append(w / beta)
    T = np.diag(a) + np.diag(b[: len(a) - 1], 1) + np.diag(b[: len(a) - 1], -1)
    return float(np.linalg.eigvalsh(T)[0]), np.array(a), np.array(b)


def ground_energy_sparse(A) -> float:
    import scipy.sparse.linalg as sla
    if A.shape[0] < 400:
        return ground_energy_dense(A)
    w = sla.eigsh(A, k=1, which="SA", tol=1e-14, maxiter=100000)[0]
    return float(w[0])


# ------------------------------------------------------------ observables
def table_from_factors(terms) -> Terms:
    """(scalar, [(code, site), ...]) physical terms -> driver tables: factors
    daggered in written order, scalar conjugated, as ComputeStaticExpValZeroT
    builds them (exact_diagonalization/HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:
    434-455).  Codes 0 Sz, 1 Sp, 2 Sm, 9 I."""
    terms = list(terms)
    C_ = max([len(f) for _, f in terms] + [1])
    dag = {0: 0, 1: 2, 2: 1, 9: 9}
    n_ops = np.zeros(len(terms), np.int32)
    codes = np.zeros(len(terms) * C_, np.int32)
    sites = np.zeros(len(terms) * C_, np.int32)
    sc = np.zeros(len(terms), np.complex128)
    for t, (s, f) in enumerate(terms):
        n_ops[t] = len(f)
        for j, (c, q) in enumerate(f):
            codes[t * C_ + j] = dag[c]
            sites[t * C_ + j] = q
        sc[t] = np.conj(s)
    return Terms(n_ops, codes, sites, sc, C_)


def expval_ref_rule(sec: Sector, terms: Terms, alpha: int, phi, with_break: bool = True,
                    tol_norm: float = 1e-5) -> complex:
    """Restatement of ExpecValArbOperatorAbelianIrrepProjHeisenbergZeroT + the
    driver's reduction (utils.cu:442-550; HeisenbergGenericXXZ_AbelianSymms_CUDA.cu:
    596-597) on phi over all R orbits.  with_break keeps the reference's exit
    from the member loop when a factor annihilates a member."""
    g = sec.group
    chars = np.ascontiguousarray(g.chars.astype(np.complex128)).view(np.float64).ravel()
    ph = np.ascontiguousarray(np.asarray(phi, np.complex128)).view(np.float64).ravel()
    out = np.zeros(2)
    lib().oc_expval_ref(g.L, g.G, np.ascontiguousarray(g.perm).ravel(), g.n_ext, sec.R, sec.reps,
                        sec.orbit, np.ascontiguousarray(sec.norms.ravel()), sec.norms.shape[1], alpha,
                        chars, tol_norm, terms.H, terms.n_col, terms.n_ops, terms.codes, terms.sites,
                        np.ascontiguousarray(terms.scalar).view(np.float64), ph, 1 if with_break else 0, out)
    return complex(out[0], out[1])


def apply_table(L: int, k: int, terms: Terms):
    """Matrix M[t, s] = <t| table |s> of the tables applied in order (the
    daggered operator) on the Sz sector in rank order."""
    states = enumerate_sector(L, k)
    pos = {int(s): i for i, s in enumerate(states)}
    M = np.zeros((len(states), len(states)), np.complex128)
    for j, s0 in enumerate(states):
        for h in range(terms.H):
            t = int(s0)
            c = complex(terms.scalar[h])
            ok = True
            for x in range(terms.n_ops[h]):
                code = terms.codes[h * terms.n_col + x]
                q = terms.sites[h * terms.n_col + x]
                spin = (t >> q) & 1
                if code == 2:
                    if not spin:
                        ok = False
                        break
                    t &= ~(1 << q)
                elif code == 1:
                    if spin:
                        ok = False
                        break
                    t |= 1 << q
                elif code == 0:
                    c *= 0.5 if spin else -0.5
            if ok and t in pos:
                M[pos[t], j] += c
    return M


def dense_operator(L: int, k: int, terms: Terms) -> np.ndarray:
    """The physical operator of driver-form tables on the Sz sector (rank
    order): the tables apply A^dagger, so A = (applied matrix)^H."""
    return apply_table(L, k, terms).conj().T


def irrep_basis(group: Group, alpha: int, k: int) -> np.ndarray:
    """Orthonormal basis (columns, Sz-sector coordinates in rank order) of the
    irrep alpha: the range of P = (1/n_ext) sum_e conj(chi_alpha(e)) U_e,
    U_e moving the spin at site q to perm[e][q] (spin-inverted for e >= G).
    This is the subspace whose lowest energy the sector's irrep alpha gives."""
    L, G = group.L, group.G
    states = enumerate_sector(L, k)
    pos = {int(s): i for i, s in enumerate(states)}
    n = len(states)
    P = np.zeros((n, n), np.complex128)
    for e in range(group.n_ext):
        c = np.conj(group.chars[alpha, e]) / group.n_ext
        row = np.ascontiguousarray(group.perm[e % G])
        for j, s0 in enumerate(states):
            t = int(lib().oc_apply(int(s0), L, row, 1 if e >= G else 0))
            if t in pos:
                P[pos[t], j] += c
    w, V = np.linalg.eigh(0.5 * (P + P.conj().T))
    return V[:, w > 0.5]


def irrep_ground_state(Hd: np.ndarray, B: np.ndarray):
    """Lowest eigenpair of Hd restricted to span(B): (E0, psi, gap)."""
    w, v = np.linalg.eigh(B.conj().T @ Hd @ B)
    return float(w[0]), B @ v[:, 0], float(w[1] - w[0]) if len(w) > 1 else np.inf


def sym_table(group: Group, terms) -> list:
    """Group average (1/n_ext) sum_e U_e^-1 A U_e of physical factor terms:
    sites mapped by perm[e % G], S+ <-> S- and Sz -> -Sz for e >= G."""
    out = []
    flip = {0: 0, 1: 2, 2: 1, 9: 9}
    for e in range(group.n_ext):
        p = group.perm[e % group.G]
        z = e >= group.G
        for s, f in terms:
            sign = (-1) ** sum(1 for c, _ in f if c == 0) if z else 1
            out.append((s * sign / group.n_ext, [((flip[c] if z else c), int(p[q])) for c, q in f]))
    return out


def expval_sym_rule(sec: Sector, terms, alpha: int, phi, tol_norm: float = 1e-5) -> complex:
    """conj(phi^H M phi) / |phi|^2 with M the symmetric-basis matrix (Hamiltonian
    rule, ell_terms) of the group-averaged operator; phi over active rows.
    Terms with unequal numbers of S+ and S- leave the Sz sector and have zero
    expectation; they are dropped before the table is built."""
    terms = [(s, f) for s, f in terms
             if sum(1 for c, _ in f if c == 1) == sum(1 for c, _ in f if c == 2)]
    if not terms:
        return 0j
    tab = table_from_factors(sym_table(sec.group, terms))
    rows = active_rows(sec, alpha, tol_norm)
    W = max(2, int(tab.H) + 1)
    rc, ind, val, tr = ell_terms(sec, tab, alpha, W, tol_norm)
    assert rc >= 0
    M = ell_to_csr(ind, val, tr, rows)
    M = M.toarray() if hasattr(M, "toarray") else np.asarray(M)
    phi = np.asarray(phi, np.complex128)
    return complex(np.conj(phi.conj() @ M @ phi) / np.vdot(phi, phi).real)


def ref_expval(sec: Sector, terms: Terms, alpha: int, phi_orbits, tol_norm: float = 1e-5) -> complex:
    """The reference's kernel itself (oracle/_ref) on phi over all R orbits,
    FP32 as in the reference.  The group must have no spin inversion."""
    g = sec.group
    assert not g.flip
    L, G, k = g.L, g.G, sec.k
    n_irr = g.chars.shape[0]
    n = binom(L, k)
    chars32 = np.ascontiguousarray(g.chars.astype(np.complex64)).view(np.float32).ravel()
    reps = np.zeros(max(n, 1), np.uint32)
    srs = np.zeros(max(n * G, 1), np.uint32)
    norms = np.zeros(max(n * n_irr, 1), np.float32)
    orbit = np.zeros(max(2 * n, 1), np.uint32)
    perm = np.ascontiguousarray(g.perm).ravel()
    R = ref().ref_build_srs_complex(L, k, G, perm, n_irr, chars32, reps, n, srs, norms, orbit)
    assert R == sec.R
    act = {0: 0, 1: 1, 2: -1}
    C_ = terms.n_col
    actions = np.zeros(terms.H * C_, np.int32)
    sites = -np.ones(terms.H * C_, np.int32)
    for h in range(terms.H):
        for x in range(terms.n_ops[h]):
            actions[h * C_ + x] = act[int(terms.codes[h * C_ + x])]
            sites[h * C_ + x] = terms.sites[h * C_ + x]
    sc = np.ascontiguousarray(terms.scalar.astype(np.complex64)).view(np.float32).ravel()
    out = np.zeros(2, np.float32)
    phi = np.asarray(phi_orbits)
    if np.iscomplexobj(phi):
        f = ref().ref_expval_complex
        ph = np.ascontiguousarray(phi.astype(np.complex64)).view(np.float32).ravel()
    else:
        f = ref().ref_expval_real
        ph = np.ascontiguousarray(phi.astype(np.float32))
    f(L, k, G, R, srs[: R * G], orbit[: 2 * n], n_irr, chars32, alpha, norms[: R * n_irr], tol_norm,
      terms.H, C_, terms.n_ops, actions, sites, sc, ph, out)
    return complex(float(out[0]), float(out[1]))
