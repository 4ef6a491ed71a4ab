"""A minimal HDF5 writer for the v7.3 reader's tests (test infrastructure).

Writes what MATLAB's v7.3 files are made of: a 512-byte MATLAB user block,
superblock version 0, groups as symbol tables (v1 B-tree, local heap, symbol
node), version-1 object headers, datasets stored contiguous or chunked (v1
B-tree) with the shuffle and deflate filters, IEEE float and compound
{real, imag} datatypes, and a MATLAB_class string attribute.  Arrays are
stored as MATLAB stores them: column-major, i.e. the HDF5 dataset is the
transpose of the MATLAB array.  Written from the HDF5 file-format
specification; the reader is pinned separately to a file MATLAB wrote.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


def _pad8(b: bytes) -> bytes:
    return b + b"\x00" * (-len(b) % 8)


class _Buf:
    def __init__(self):
        self.b = bytearray()

    def alloc(self, n: int) -> int:
        n += -n % 8
        off = len(self.b)
        self.b += b"\x00" * n
        return off

    def put(self, off: int, data: bytes) -> None:
        self.b[off:off + len(data)] = data

    def add(self, data: bytes) -> int:
        off = self.alloc(len(data))
        self.put(off, data)
        return off


def _float_type(itemsize: int) -> bytes:
    if itemsize == 8:
        sign, prec, eloc, esz, msz, bias = 63, 64, 52, 11, 52, 1023
    else:
        sign, prec, eloc, esz, msz, bias = 31, 32, 23, 8, 23, 127
    bits = 0x20 | (sign << 8)
    return (bytes([0x11]) + bits.to_bytes(3, "little") + struct.pack("<I", itemsize)
            + struct.pack("<HHBBBBI", 0, prec, eloc, esz, 0, msz, bias))


def _datatype(dt: np.dtype) -> bytes:
    if dt.kind == "c":
        half = dt.itemsize // 2
        ft = _float_type(half)
        out = bytes([0x16]) + (2).to_bytes(3, "little") + struct.pack("<I", dt.itemsize)
        for name, off in (("real", 0), ("imag", half)):
            out += _pad8(name.encode() + b"\x00") + struct.pack("<I", off) + b"\x00" * 28 + ft
        return out
    if dt.kind == "f":
        return _float_type(dt.itemsize)
    raise ValueError(f"unsupported dtype {dt}")


def _dataspace(shape) -> bytes:
    return bytes([1, len(shape), 0, 0]) + b"\x00" * 4 + b"".join(struct.pack("<Q", d) for d in shape)


def _message(mtype: int, data: bytes) -> bytes:
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), 0) + data


def _object_header(buf: _Buf, msgs: list[bytes]) -> int:
    body = b"".join(msgs)
    head = struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\x00" * 4
    return buf.add(head + body)


def _attr_string(name: str, value: str) -> bytes:
    nm = name.encode() + b"\x00"
    val = value.encode()
    dt = bytes([0x13]) + (0).to_bytes(3, "little") + struct.pack("<I", len(val))
    ds = bytes([1, 0, 0, 0]) + b"\x00" * 4
    return (struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(ds)) + _pad8(nm) + _pad8(dt) + _pad8(ds) + val)


def _dataset(buf: _Buf, arr: np.ndarray, chunks=None, deflate: int = 0, shuffle: bool = False) -> int:
    """arr in HDF5 order (already transposed from MATLAB's)."""
    arr = np.ascontiguousarray(arr)
    if arr.dtype.kind == "c":
        st = np.empty(arr.shape, np.dtype([("real", arr.real.dtype), ("imag", arr.real.dtype)]))
        st["real"], st["imag"] = arr.real, arr.imag
        raw_arr = st
    else:
        raw_arr = arr
    isz = raw_arr.dtype.itemsize
    msgs = [_message(0x01, _dataspace(arr.shape)), _message(0x03, _datatype(arr.dtype))]
    if chunks is None:
        data_off = buf.add(raw_arr.tobytes())
        msgs.append(_message(0x08, bytes([3, 1]) + struct.pack("<QQ", data_off, raw_arr.nbytes)))
    else:
        rank = arr.ndim
        entries = []
        for idx in np.ndindex(*[-(-s // c) for s, c in zip(arr.shape, chunks)]):
            offs = [i * c for i, c in zip(idx, chunks)]
            block = np.zeros(chunks, raw_arr.dtype)
            src = raw_arr[tuple(slice(o, o + c) for o, c in zip(offs, chunks))]
            block[tuple(slice(0, s) for s in src.shape)] = src
            raw = block.tobytes()
            if shuffle:
                raw = np.frombuffer(raw, np.uint8).reshape(-1, isz).T.tobytes()
            if deflate:
                raw = zlib.compress(raw, deflate)
            entries.append((offs, buf.add(raw), len(raw)))
        ksz = 8 + 8 * (rank + 1)
        node = bytearray(b"TREE" + bytes([1, 0]) + struct.pack("<H", len(entries)) + struct.pack("<QQ", UNDEF, UNDEF))
        for offs, addr, size in entries:
            node += struct.pack("<II", size, 0) + b"".join(struct.pack("<Q", o) for o in offs + [0])
            node += struct.pack("<Q", addr)
        node += struct.pack("<II", 0, 0) + b"".join(struct.pack("<Q", s) for s in list(arr.shape) + [0])
        assert len(node) == 24 + len(entries) * (ksz + 8) + ksz
        bt = buf.add(bytes(node))
        msgs.append(_message(0x08, bytes([3, 2, rank + 1]) + struct.pack("<Q", bt)
                             + b"".join(struct.pack("<I", c) for c in list(chunks) + [isz])))
        filt = []
        if shuffle:
            filt.append(struct.pack("<HHHH", 2, 0, 0, 1) + struct.pack("<I", isz) + b"\x00" * 4)
        if deflate:
            filt.append(struct.pack("<HHHH", 1, 0, 0, 1) + struct.pack("<I", deflate) + b"\x00" * 4)
        if filt:
            msgs.append(_message(0x0B, bytes([1, len(filt)]) + b"\x00" * 6 + b"".join(filt)))
    cls = {"f": "double" if arr.real.dtype.itemsize == 8 else "single"}.get(arr.real.dtype.kind, "double")
    msgs.append(_message(0x0C, _attr_string("MATLAB_class", cls)))
    return _object_header(buf, msgs)


def _group(buf: _Buf, children: dict) -> int:
    """children: {name: object header address}; returns the group's header address."""
    names = sorted(children)
    heap_data = bytearray(b"\x00" * 8)  # offset 0: the empty name
    name_off = {}
    for n in names:
        name_off[n] = len(heap_data)
        heap_data += _pad8(n.encode() + b"\x00")
    heap_data_addr = buf.add(bytes(heap_data))
    heap = buf.add(b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap_data), UNDEF, heap_data_addr))
    snod = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(names)))
    for n in names:
        snod += struct.pack("<QQII", name_off[n], children[n], 0, 0) + b"\x00" * 16
    snod_addr = buf.add(bytes(snod))
    last = name_off[names[-1]] if names else 0
    tree = b"TREE" + bytes([0, 0]) + struct.pack("<H", 1) + struct.pack("<QQ", UNDEF, UNDEF)
    tree += struct.pack("<QQQ", 0, snod_addr, last)
    bt = buf.add(tree)
    return _object_header(buf, [_message(0x11, struct.pack("<QQ", bt, heap))])


def write_mat73(path: str, variables: dict, chunks: dict | None = None, deflate: int = 6,
                shuffle: bool = True) -> None:
    """variables: {name: MATLAB-order array, or {name: ...} for a group}.
    chunks: {name: MATLAB-order chunk shape} for the datasets to store chunked
    (with shuffle + deflate), the rest contiguous."""
    chunks = chunks or {}
    buf = _Buf()
    sb = buf.alloc(96)  # superblock v0 with the root symbol-table entry

    def emit(name, v):
        if isinstance(v, dict):
            return _group(buf, {k: emit(k, x) for k, x in v.items()})
        a = np.asarray(v)
        ch = chunks.get(name)
        return _dataset(buf, a.T, tuple(reversed(ch)) if ch else None, deflate if ch else 0, shuffle and bool(ch))

    root = _group(buf, {k: emit(k, v) for k, v in variables.items()})
    sig = b"\x89HDF\r\n\x1a\n"
    head = sig + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0)
    head += struct.pack("<QQQQ", 512, UNDEF, len(buf.b) + 512, UNDEF)
    head += struct.pack("<QQII", 0, root, 0, 0) + b"\x00" * 16
    assert len(head) == 96
    buf.put(sb, head)
    user = b"MATLAB 7.3 MAT-file, written by tests/h5write.py, HDF5 schema 1.00 ."
    user = user.ljust(116, b" ") + b"\x00" * 8 + b"\x00\x02IM"
    user = user.ljust(512, b"\x00")
    with open(path, "wb") as f:
        f.write(user + bytes(buf.b))
