"""Sector and matrix table files on the GPU.

A save -> load round trip is bit-exact: representatives, norms, active rows
and the orbit map of the sector; H*v in FP64 and FP32 from the stored
values; the matrix-free product from the stored term tables; Lanczos
energies.  Loading a matrix into another sector or irrep is refused, and so
are stored representatives that are not orbit minima of the group."""
import numpy as np
import pytest

import qmbcuda_b200 as q
from helpers import sector_cases
from qmbcuda_b200 import tablefile as TF

pytestmark = pytest.mark.gpu
A = q._capi
CASES = [c for c in sector_cases() if c[0] in ("chain12_T", "chain12_TZ", "square4x4_C4")]


def _sector(case, a=1):
    name, L, k, perm, ch, flip, bonds = case
    s = q.Sector(L, k, perm, spin_flip=flip).set_irrep(ch[a % len(ch)])
    return s


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sector_round_trip(tmp_path, case):
    s = _sector(case)
    p = str(tmp_path / "s.qmbt")
    s.save(p)
    s2 = q.Sector.load(p)
    i1, i2 = s.info, s2.info
    assert (i1.n_states, i1.n_orbits, i1.n_active, i1.n_ext, i1.structured, i1.is_real) == \
           (i2.n_states, i2.n_orbits, i2.n_active, i2.n_ext, i2.structured, i2.is_real)
    assert np.array_equal(s.reps(), s2.reps())
    assert np.array_equal(s.norms().view(np.uint64), s2.norms().view(np.uint64))
    assert np.array_equal(s.active(), s2.active())
    assert np.array_equal(s.orbit_map(), s2.orbit_map())


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("jxy", [1.0, 0.8 + 0.3j])
def test_ham_round_trip(tmp_path, case, jxy):
    name, L, k, perm, ch, flip, bonds = case
    s = _sector(case)
    terms = q.xxz_terms(bonds, jxy, 0.6)
    h = q.Hamiltonian(s, terms)
    ps, ph = str(tmp_path / "s.qmbt"), str(tmp_path / "h.qmbt")
    s.save(ps)
    h.save(ph)
    s2 = q.Sector.load(ps)
    h2 = q.Hamiltonian.load(s2, ph)
    i1, i2 = h.info, h2.info
    assert (i1.n_rows, i1.nnz_offdiag, i1.padded, i1.max_row, i1.is_complex) == \
           (i2.n_rows, i2.nnz_offdiag, i2.padded, i2.max_row, i2.is_complex)
    rng = np.random.default_rng(1)
    for prec in (A.PREC_FP64, A.PREC_FP32):
        dt = h.dtype(prec)
        x = rng.standard_normal(i1.n_rows).astype(dt)
        if np.iscomplexobj(x):
            x = x + 1j * rng.standard_normal(i1.n_rows).astype(dt)
        y1, y2 = h.hv_host(x, prec), h2.hv_host(x, prec)
        assert np.array_equal(y1.view(np.uint8), y2.view(np.uint8)), prec
    for hv in (A.HV_STORED, A.HV_MATRIX_FREE):
        # the two handles must run identical solves, converged or not
        r1 = h.lanczos(mode=A.MODE_FP64, max_iter=300, tol=1e-12, hv=hv, allow_unconverged=True)
        r2 = h2.lanczos(mode=A.MODE_FP64, max_iter=300, tol=1e-12, hv=hv, allow_unconverged=True)
        assert r1.E0 == r2.E0 and r1.iters == r2.iters, hv


def test_ham_load_refuses_other_sector_or_irrep(tmp_path):
    case = CASES[0]
    name, L, k, perm, ch, flip, bonds = case
    s = _sector(case, 1)
    h = q.Hamiltonian(s, q.xxz_terms(bonds, 1.0, 0.6))
    ph = str(tmp_path / "h.qmbt")
    h.save(ph)
    other = _sector(case, 2)
    with pytest.raises(q.QMBError) as e:
        q.Hamiltonian.load(other, ph)
    assert e.value.status == A.QMB_ERR_INVALID and "irrep" in str(e.value)
    s3 = q.Sector(L, k - 1, perm).set_irrep(ch[1])
    with pytest.raises(q.QMBError) as e:
        q.Hamiltonian.load(s3, ph)
    assert e.value.status == A.QMB_ERR_INVALID
    b = bytearray(open(ph, "rb").read())
    b[-8] ^= 1
    open(ph, "wb").write(bytes(b))
    with pytest.raises(q.QMBError) as e:
        q.Hamiltonian.load(s, ph)
    assert e.value.status == A.QMB_ERR_CORRUPT


def test_sector_load_refuses_non_minimal_reps(tmp_path):
    """A file with valid checksums whose representatives include a string
    that is not its orbit's minimum (the sector's largest string)."""
    case = CASES[0]
    name, L, k, perm, ch, flip, bonds = case
    s = _sector(case)
    p = str(tmp_path / "s.qmbt")
    s.save(p)
    kind, ver, meta, secs = TF.read(p)
    reps = np.frombuffer(secs[TF.TAGS["reps"]][1], np.uint64)
    top = np.uint64(((1 << k) - 1) << (L - k))
    bad = np.concatenate([reps, [top]])
    meta[4] = len(bad)
    TF.write(p, kind, meta, [(TF.TAGS["perm"], np.frombuffer(secs[TF.TAGS["perm"]][1], np.uint32)),
                             (TF.TAGS["reps"], bad),
                             (TF.TAGS["chars"], np.frombuffer(secs[TF.TAGS["chars"]][1], np.complex128))])
    with pytest.raises(q.QMBError) as e:
        q.Sector.load(p)
    assert e.value.status == A.QMB_ERR_INVALID and "orbit minima" in str(e.value)
