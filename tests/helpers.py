"""Shared builders for the tests: the same sector / Hamiltonian built through
the product (C ABI) and through the oracle (CPU restatement)."""
import numpy as np

import oracle as O
import qmbcuda_b200 as q


def oracle_terms(t: q.TermTable) -> O.Terms:
    return O.Terms(t.n_ops, np.ascontiguousarray(t.codes.ravel()),
                   np.ascontiguousarray(t.sites.ravel()), t.scalar, t.codes.shape[1])


def oracle_group(perm, chars_table, flip=False) -> O.Group:
    perm = np.ascontiguousarray(np.atleast_2d(perm), np.uint32)
    ch = np.atleast_2d(np.asarray(chars_table, np.complex128))
    return O.Group(perm.shape[1], perm, ch, flip)


def rotations_4x4(n=4):
    """C4 about the centre of a 4x4 square lattice (open geometry)."""
    g = q.geometry(4, 4)
    L = 16
    R1 = np.zeros(L)
    R2 = np.zeros(L)
    q.check(q.lib().qmb_geometry_sites(g, q._capi.ptr(R1), q._capi.ptr(R2)))
    R0 = np.array([R1.mean(), R2.mean()])
    perm = np.zeros((n, L), np.uint32)
    ch = np.zeros(2 * n * n)
    q.check(q.lib().qmb_group_rotations(L, q._capi.ptr(R1), q._capi.ptr(R2), n, q._capi.ptr(R0),
                                        q._capi.ptr(perm), q._capi.ptr(ch)))
    return perm, ch.view(np.complex128).reshape(n, n)


# (name, L, n_up, perm, chars_table, flip, bonds)
def sector_cases():
    cases = []
    p, ch = q.translation_group(12)
    cases.append(("chain12_T", 12, 6, p, ch, False, q.chain_bonds(12)))
    p, ch = q.translation_group(12)
    chf = np.block([[ch, ch], [ch, -ch]])
    cases.append(("chain12_TZ", 12, 6, p, chf, True, q.chain_bonds(12)))
    p, ch = q.translation_group(10)
    cases.append(("chain10_T_nup3", 10, 3, p, ch, False, q.chain_bonds(10) + q.chain_bonds(10, 2)))
    p, ch = q.translation_group(4, 4)
    cases.append(("square4x4_T", 16, 8, p, ch, False, q.square_bonds(4, 4)))
    p, ch = rotations_4x4()
    cases.append(("square4x4_C4", 16, 8, p, ch, False, q.square_bonds(4, 4)))
    p = np.arange(10, dtype=np.uint32)[None, :]
    cases.append(("trivial10", 10, 4, p, np.ones((1, 1)), False, q.chain_bonds(10)))
    return cases
