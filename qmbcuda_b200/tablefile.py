"""Reader and writer of the table-file format in pure Python (numpy), for
tools that do not load libqmb_b200.so.  The library's own implementation is
qmbcuda_b200/csrc/qmb_store.cu; both follow this layout (little-endian):

  header, 256 bytes   magic b"QMBTABLE", u32 version (1), u32 kind
                      (1 sector, 2 matrix, 3 reference ELL), u32 section
                      count, u32 byte-order mark 0x01020304, u64 meta[27],
                      u64 checksum of the section table, u64 checksum of the
                      header with this last field zero
  section table       per section: u32 tag, u32 element bytes, u64 count,
                      u64 offset, u64 checksum of the payload
  payloads            at 64-byte aligned offsets

checksum(b): h = 0xcbf29ce484222325 ^ len(b); for every 8-byte little-endian
word w (the tail zero-padded): h = (h ^ w) * 0x100000001b3 mod 2^64,
h ^= h >> 29.
"""
from __future__ import annotations

import os
import struct

import numpy as np

MAGIC = b"QMBTABLE"
VERSION = 1
BYTE_ORDER = 0x01020304
KIND_SECTOR, KIND_HAM, KIND_REF_ELL = 1, 2, 3
TAGS = {"perm": 1, "reps": 2, "chars": 3,
        "slice_off": 16, "slice_w": 17, "col": 18, "val64": 19, "val32": 20, "diag64": 21, "diag32": 22,
        "t_nops": 23, "t_ops": 24, "t_scalar": 25,
        "ind": 32, "val": 33, "track": 34}
_HDR = struct.Struct("<8s4I27Q2Q")
_ENT = struct.Struct("<2I3Q")
_M64 = (1 << 64) - 1


def checksum(b: bytes) -> int:
    n = len(b)
    h = 0xCBF29CE484222325 ^ n
    pad = (-n) % 8
    words = np.frombuffer(bytes(b) + b"\0" * pad, dtype="<u8")
    for w in words.tolist():
        h = ((h ^ w) * 0x100000001B3) & _M64
        h ^= h >> 29
    return h


def write(path: str, kind: int, meta, sections) -> None:
    """sections: list of (tag, numpy array); element size = array itemsize."""
    meta = list(meta) + [0] * (27 - len(meta))
    table, blobs = [], []
    off = (_HDR.size + _ENT.size * len(sections) + 63) // 64 * 64
    for tag, arr in sections:
        a = np.ascontiguousarray(arr)
        b = a.tobytes()
        table.append((tag, a.itemsize, a.size, off, checksum(b)))
        blobs.append((off, b))
        off = (off + len(b) + 63) // 64 * 64
    tab = b"".join(_ENT.pack(*e) for e in table)
    hd = _HDR.pack(MAGIC, VERSION, kind, len(sections), BYTE_ORDER, *meta, checksum(tab), 0)
    hd = _HDR.pack(MAGIC, VERSION, kind, len(sections), BYTE_ORDER, *meta, checksum(tab), checksum(hd))
    out = bytearray(off)
    out[:len(hd)] = hd
    out[len(hd):len(hd) + len(tab)] = tab
    for o, b in blobs:
        out[o:o + len(b)] = b
    tmp = f"{path}.tmp.{os.getpid()}"
    with open(tmp, "wb") as f:
        f.write(bytes(out))
    os.replace(tmp, path)


def read(path: str, verify: bool = True):
    """(kind, version, meta[27], {tag: (element bytes, raw bytes)})."""
    data = open(path, "rb").read()
    if len(data) < _HDR.size:
        raise ValueError("shorter than a header")
    f = _HDR.unpack_from(data, 0)
    magic, version, kind, n_sec, order = f[:5]
    meta, tab_sum, hdr_sum = list(f[5:32]), f[32], f[33]
    if magic != MAGIC or order != BYTE_ORDER:
        raise ValueError("not a table file of this byte order")
    if verify and checksum(data[:_HDR.size - 8] + b"\0" * 8) != hdr_sum:
        raise ValueError("header checksum mismatch")
    tab = data[_HDR.size:_HDR.size + _ENT.size * n_sec]
    if verify and checksum(tab) != tab_sum:
        raise ValueError("section table checksum mismatch")
    secs = {}
    for i in range(n_sec):
        tag, es, count, off, s = _ENT.unpack_from(tab, _ENT.size * i)
        b = data[off:off + es * count]
        if len(b) != es * count:
            raise ValueError("section runs past the end of the file")
        if verify and checksum(b) != s:
            raise ValueError(f"checksum mismatch in section {tag}")
        secs[tag] = (es, b)
    return kind, version, meta, secs
