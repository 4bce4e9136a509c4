"""The XY/Z split of XXZ term tables that batched solves rely on
(H = c_xy A + c_z D), checked on the host through the oracle: for every
momentum sector of an L=10 chain, A(part="xy") has no diagonal, D(part="z")
is diagonal, and c_xy A + c_z D equals the matrix of the full table with
couplings c_xy, c_z for real c_xy; with a complex c_xy the full matrix
stays Hermitian."""
import numpy as np
import pytest

import oracle as O
import qmbcuda_b200 as q
from helpers import oracle_group, oracle_terms


def _matrix(sec, t, a):
    rc, ind, val, tr = O.ell_terms(sec, oracle_terms(t), a, 2 * t.n_terms + 1)
    return O.ell_to_csr(ind, val, tr, O.active_rows(sec, a)).toarray()


@pytest.mark.parametrize("cxy,cz", [(1.0, 0.0), (0.8, 1.3), (0.7 + 0.2j, -0.4)])
def test_xy_z_split_sums_to_full(cxy, cz):
    L = 10
    perm, ch = q.translation_group(L)
    sec = O.build_sector(oracle_group(perm, ch), L // 2)
    bonds = q.chain_bonds(L)
    txy = q.xxz_terms(bonds, 1.0, 0.0, part="xy")
    tz = q.xxz_terms(bonds, 0.0, 1.0, part="z")
    full = q.xxz_terms(bonds, cxy, cz)
    assert txy.n_terms == 2 * L and tz.n_terms == L and full.n_terms == 3 * L
    for a in range(L):
        if len(O.active_rows(sec, a)) == 0:
            continue
        Axy, Dz, H = _matrix(sec, txy, a), _matrix(sec, tz, a), _matrix(sec, full, a)
        assert np.allclose(np.diag(Axy), 0.0)
        assert np.allclose(Dz, np.diag(np.diag(Dz)))
        # the batched form scales the unit tables; a complex c_xy scales the
        # hopping towards one site and its conjugate the other way, so it
        # only matches for real c_xy
        if np.isreal(cxy):
            assert np.allclose(cxy.real * Axy + cz * Dz, H, atol=1e-12)
        assert np.allclose(H, H.conj().T, atol=1e-12)
