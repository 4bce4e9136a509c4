"""Writes tests/golden/reference_tables.npz: outputs of the reference's own
code, compiled for the host from its unmodified sources into oracle/_ref
(oracle/Makefile), on small fixed inputs.  The tests compare the oracle and
the engine with these arrays, so the pin to the reference holds where the
reference sources are not present.

    make -C oracle          # needs the reference sources
    python tests/golden/make_golden.py

Contents (key prefix = case):
  <case>_reps, _orbit, _norms     SetUpSRS / SolveSRS_min / ComputeSRSNorms /
                                  ComputeOrbitIndices tables (rank of each
                                  representative, orbit map, FP32 norms [R][NIr])
  <case>_a<a>_ind/_val/_track     BuildHamiltonianXXZForAbelianGroup ELL of the
                                  XXZ terms J_xy = 1 + 0.3i, J_z = 0.6 on the
                                  case's bonds, irrep a, with the reference norms
  tstd_<geom>_ti/_tj/_tv          T_standard pair lists
  hv_x, hv_y                      SparseMatDenseVec_prod_EEL_host on the L=12
                                  k=0 ELL (Heisenberg chain) and a seeded x
  e0_chain12                      dense FP64 ground energies of the 12 momentum
                                  irreps of the L=12 Heisenberg chain (oracle)
  ev_chain10_a<a>_phi             FP32 ground state over all orbits of irrep a of
                                  the L=10 Heisenberg chain (oracle ELL, dense)
  ev_chain10_a<a>_<op>            ExpecValArbOperatorAbelianIrrepProjHeisenbergZeroT
                                  + reduction / G on that state, operators EV_OPS
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

CASES = [("chain10", lambda: O.translation_group(10), 5, "chain"),
         ("square2x4", lambda: O.translation_group(2, 4), 4, "ring")]
TSTD = [("chain16", 16, 1, 1, (1.0, 0.0, 0.0, 1.0), [1.0], [1.0001], 1, 1),
        ("square2x4_pbc", 2, 4, 1, (1.0, 0.0, 0.0, 1.0), [1.0, 0.15 + 0.15j], [1.0001, 1.4143], 1, 1)]


# Operators of the expectation-value fixtures: (scalar, [(code, site), ...])
# with codes 0 Sz, 1 Sp, 2 Sm, factors in written order.
EV_OPS = {
    "SzSz03": [(1.0, [(0, 0), (0, 3)])],
    "SzSz01i": [(1j, [(0, 0), (0, 1)])],
    "Sz2": [(1.0, [(0, 2)])],
    "SzSzSzSz": [(2.0, [(0, 0), (0, 1), (0, 4), (0, 7)])],
    "SpSm01": [(1.0, [(1, 0), (2, 1)])],
    "SpSm02hc": [(0.5, [(1, 0), (2, 2)]), (0.5, [(2, 0), (1, 2)])],
}
EV_IRREPS = (0, 5, 1, 3)


def ev_state(sec, a):
    """Lowest eigenvector of irrep a of the L=10 Heisenberg chain over all R
    orbits (zero on null orbits), normalised, as FP32 complex."""
    t = O.xxz_terms(O.chain_bonds(sec.group.L), 1.0, 1.0)
    rows = O.active_rows(sec, a)
    rc, ind, val, tr = O.ell_terms(sec, t, a, 2 * sec.group.L + 1)
    M = O.ell_to_csr(ind, val, tr, rows)
    M = M.toarray() if hasattr(M, "toarray") else np.asarray(M)
    w, V = np.linalg.eigh(M)
    v = V[:, 0] / V[np.argmax(np.abs(V[:, 0])), 0] * np.abs(V[:, 0]).max()
    phi = np.zeros(sec.R, np.complex128)
    phi[rows] = v / np.linalg.norm(v)
    return phi.astype(np.complex64)


def ref_srs(R, g, k):
    L, G = g.L, g.G
    N = O.binom(L, k)
    reps = np.zeros(N, np.uint32)
    srs = np.zeros(N * G, np.uint32)
    n_irr = g.chars.shape[0]
    norms = np.zeros(N * n_irr, np.float32)
    oi = np.zeros(2 * N, np.uint32)
    ch = np.ascontiguousarray(g.chars.astype(np.complex64)).view(np.float32).ravel()
    Rn = R.ref_build_srs_complex(L, k, G, np.ascontiguousarray(g.perm), n_irr, ch, reps, N, srs, norms, oi)
    return Rn, reps[:Rn].copy(), srs[: Rn * G].copy(), norms[: Rn * n_irr].reshape(Rn, n_irr).copy(), oi


def bonds_of(kind, L):
    return O.chain_bonds(L) if kind == "chain" else [(i, (i + 1) % L) for i in range(L)]


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref is not built (needs the reference sources): run make -C oracle")
    R = O.ref()
    out = {}
    for name, mk, k, kind in CASES:
        g = mk()
        Rn, reps, srs, norms, oi = ref_srs(R, g, k)
        out[f"{name}_reps"], out[f"{name}_orbit"], out[f"{name}_norms"] = reps, oi, norms
        t = O.xxz_terms(bonds_of(kind, g.L), 1.0 + 0.3j, 0.6)
        W = 2 * len(bonds_of(kind, g.L)) + 1
        n_irr = g.chars.shape[0]
        ch = np.ascontiguousarray(g.chars.astype(np.complex64)).view(np.float32).ravel()
        sc = np.ascontiguousarray(t.scalar.astype(np.complex64)).view(np.float32).ravel()
        for a in sorted({0, 1, n_irr // 2}):
            ind = np.zeros(Rn * W, np.uint32)
            val = np.zeros(2 * Rn * W, np.float32)
            tr = np.zeros(Rn, np.int16)
            R.ref_ham_terms_complex(g.L, k, g.G, Rn, srs, oi, n_irr, ch, a, norms.ravel().copy(), 1e-5,
                                    t.H, t.n_col, t.n_ops, t.codes, t.sites, sc, W, ind, val, tr)
            out[f"{name}_a{a}_ind"] = ind.reshape(Rn, W)
            out[f"{name}_a{a}_val"] = val.view(np.complex64).reshape(Rn, W)
            out[f"{name}_a{a}_track"] = tr
    for name, N1, N2, M, A4, J, rg, intra, inter in TSTD:
        cap = 4000
        ti = np.zeros(cap, np.int32); tj = np.zeros(cap, np.int32); tv = np.zeros(2 * cap, np.float32)
        L = N1 * N2 * M
        r1 = np.zeros(L, np.float32); r2 = np.zeros(L, np.float32)
        n = R.ref_tstandard_complex(N1, N2, M, np.asarray(A4, np.float32), np.zeros(M, np.float32),
                                    np.zeros(M, np.float32), len(J),
                                    np.ascontiguousarray(np.asarray(J, np.complex64)).view(np.float32),
                                    np.asarray(rg, np.float32), intra, inter, cap, ti, tj, tv, r1, r2)
        out[f"tstd_{name}_ti"], out[f"tstd_{name}_tj"] = ti[:n], tj[:n]
        out[f"tstd_{name}_tv"] = tv[: 2 * n].view(np.complex64)
    # the reference's host H*v
    g = O.translation_group(12)
    sec = O.build_sector(g, 6)
    t = O.xxz_terms(O.chain_bonds(12), 1.0, 1.0)
    W = 25
    rc, ind, val, tr = O.ell_terms(sec, t, 0, W)
    x = np.random.default_rng(0).standard_normal(sec.R).astype(np.float32)
    y = np.zeros(sec.R, np.float32)
    R.ref_spmv_host(np.ascontiguousarray(ind.ravel()), np.ascontiguousarray(val.real.astype(np.float32).ravel()),
                    tr, x, y, sec.R, W, 1)
    out["hv_x"], out["hv_y"] = x, y
    # dense FP64 ground energies of the L=12 chain irreps
    e0 = []
    for a in range(12):
        rc, ind, val, tr = O.ell_terms(sec, t, a, W)
        rows = O.active_rows(sec, a)
        e0.append(O.ground_energy_dense(O.ell_to_csr(ind, val, tr, rows)) if len(rows) else np.nan)
    out["e0_chain12"] = np.array(e0)
    # expectation values through the reference's kernel
    g = O.translation_group(10)
    sec = O.build_sector(g, 5)
    for a in EV_IRREPS:
        phi = ev_state(sec, a)
        out[f"ev_chain10_a{a}_phi"] = phi
        real = not np.any(phi.imag)
        for nm, terms in EV_OPS.items():
            v = O.ref_expval(sec, O.table_from_factors(terms), a, phi.real if real else phi)
            out[f"ev_chain10_a{a}_{nm}"] = np.complex64(v)
    path = os.path.join(HERE, "reference_tables.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
