"""Table files without a GPU: reference-layout ELL tables through the C ABI
(qmb_ref_ell_save / qmb_ref_ell_load are host-only), the pure-Python reader
and writer against the library, and the error paths (missing file, wrong
kind, corruption, truncation, newer version).  Round trips are bit-exact."""
import os

import numpy as np
import pytest

import oracle as O
import qmbcuda_b200 as q
from qmbcuda_b200 import tablefile as TF

A = q._capi


def _ref_tables(cplx=False):
    g = O.translation_group(12)
    sec = O.build_sector(g, 6)
    t = O.xxz_terms(O.chain_bonds(12), 1.0 + (0.25j if cplx else 0.0), 0.7)
    rc, ind, val, tr = O.ell_terms(sec, t, 1 if cplx else 0, 25)
    v = val.astype(np.complex64) if cplx else val.real.astype(np.float32)
    return ind.reshape(sec.R, 25), v.reshape(sec.R, 25), tr


@pytest.mark.parametrize("cplx", [False, True])
def test_ref_ell_round_trip(tmp_path, cplx):
    ind, val, tr = _ref_tables(cplx)
    p = str(tmp_path / "ell.qmbt")
    q.save_ref_ell(p, ind, val, tr)
    i2, v2, t2 = q.load_ref_ell(p)
    assert np.array_equal(i2, ind) and np.array_equal(t2, tr)
    assert v2.dtype == val.dtype and np.array_equal(v2.view(np.uint8), val.view(np.uint8))
    # the independent reader sees the same tables
    kind, ver, meta, secs = TF.read(p)
    assert (kind, ver, meta[0], meta[1], meta[2]) == (TF.KIND_REF_ELL, 1, ind.shape[0], 25, int(cplx))
    assert np.array_equal(np.frombuffer(secs[TF.TAGS["ind"]][1], np.uint32).reshape(ind.shape), ind)
    assert np.array_equal(np.frombuffer(secs[TF.TAGS["track"]][1], np.int16), tr)
    assert not [f for f in os.listdir(tmp_path) if ".tmp." in f]


def test_python_writer_read_by_library(tmp_path):
    ind, val, tr = _ref_tables()
    p = str(tmp_path / "py.qmbt")
    TF.write(p, TF.KIND_REF_ELL, [ind.shape[0], ind.shape[1], 0],
             [(TF.TAGS["ind"], ind), (TF.TAGS["val"], val), (TF.TAGS["track"], tr)])
    i2, v2, t2 = q.load_ref_ell(p)
    assert np.array_equal(i2, ind) and np.array_equal(v2, val) and np.array_equal(t2, tr)


def _status(fn, *a):
    with pytest.raises(q.QMBError) as e:
        fn(*a)
    return e.value.status


def test_error_paths(tmp_path):
    ind, val, tr = _ref_tables()
    p = str(tmp_path / "ell.qmbt")
    q.save_ref_ell(p, ind, val, tr)
    raw = open(p, "rb").read()
    assert _status(q.load_ref_ell, str(tmp_path / "missing.qmbt")) == A.QMB_ERR_IO
    # a flipped payload byte, a flipped header byte, a truncated file
    for pos in (len(raw) - 100, 40):
        b = bytearray(raw)
        b[pos] ^= 0x10
        open(p, "wb").write(bytes(b))
        assert _status(q.load_ref_ell, p) == A.QMB_ERR_CORRUPT
    open(p, "wb").write(raw[: len(raw) // 2])
    assert _status(q.load_ref_ell, p) == A.QMB_ERR_CORRUPT
    open(p, "wb").write(b"not a table file at all" * 20)
    assert _status(q.load_ref_ell, p) == A.QMB_ERR_CORRUPT
    # a newer format version (checksums valid) is refused as unsupported
    TF.write(p, TF.KIND_REF_ELL, [ind.shape[0], ind.shape[1], 0],
             [(TF.TAGS["ind"], ind), (TF.TAGS["val"], val), (TF.TAGS["track"], tr)])
    b = bytearray(open(p, "rb").read())
    b[8:12] = (2).to_bytes(4, "little")
    hd = bytes(b[:248]) + b"\0" * 8
    b[248:256] = TF.checksum(hd).to_bytes(8, "little")
    open(p, "wb").write(bytes(b))
    assert _status(q.load_ref_ell, p) == A.QMB_ERR_UNSUPPORTED
    # a file of another kind
    TF.write(p, TF.KIND_SECTOR, [12, 6, 1, 0, 1], [(TF.TAGS["perm"], np.arange(12, dtype=np.uint32))])
    assert _status(q.load_ref_ell, p) == A.QMB_ERR_INVALID
    # a directory that does not exist
    assert _status(q.save_ref_ell, str(tmp_path / "no" / "dir.qmbt"), ind, val, tr) == A.QMB_ERR_IO


def test_checksum_matches_library(tmp_path):
    """The Python checksum is the library's: a file written by the library
    verifies in the Python reader for odd payload lengths too."""
    ind = np.arange(7 * 3, dtype=np.uint32).reshape(7, 3)
    val = np.linspace(-1, 1, 21, dtype=np.float32).reshape(7, 3)
    tr = np.array([1, 2, 3, 3, 2, 1, 0], np.int16)  # 14 bytes: a partial last word
    p = str(tmp_path / "small.qmbt")
    q.save_ref_ell(p, ind, val, tr)
    TF.read(p, verify=True)
