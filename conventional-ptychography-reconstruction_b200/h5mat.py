"""Read MATLAB v7.3 .mat files (HDF5) without h5py.

utils/io.py:25-69 reads v7.3 files with h5py, which this environment does
not have.  This module reads the subset of HDF5 that MATLAB writes for
numeric data, with NumPy and zlib only:

* superblock versions 0-3 (after a MATLAB 512-byte user block or at 0);
* object headers version 1 and 2, with continuation blocks;
* groups as symbol tables (v1 B-tree + local heap + symbol nodes) or as
  compact link messages (dense link storage in a fractal heap is refused);
* datasets with contiguous, compact or chunked (v1 B-tree) layout, the
  deflate and shuffle filters;
* fixed-point, floating-point and compound datatypes (MATLAB stores complex
  arrays as the compound {real, imag});
* attributes with fixed-point, floating-point or string values
  (MATLAB_class, MATLAB_complex).

`read_mat73(path, key=None)` returns what utils/io.py:read_data returns on
that branch: {name: array} with every array transposed from HDF5's
row-major storage back to MATLAB's dimension order, compound {real, imag}
and groups holding 'real' and 'imag' turned into complex arrays, other
groups into dicts, and names starting with '#' (MATLAB's #refs#) skipped.
Everything else (cell arrays, object references, strings as data) raises
NotImplementedError with what was found.
"""
from __future__ import annotations

import mmap
import struct
import zlib

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(ValueError):
    pass


class _File:
    def __init__(self, data: bytes):
        self.d = data
        self.sb = self._find_superblock()
        self._superblock()

    # -- primitives -----------------------------------------------------------
    def u(self, off: int, n: int) -> int:
        if off < 0 or off + n > len(self.d):
            raise H5Error(f"read of {n} bytes at {off} past the end of the file ({len(self.d)})")
        return int.from_bytes(self.d[off:off + n], "little")

    def addr(self, off: int) -> int:
        return self.u(off, self.so)

    def length(self, off: int) -> int:
        return self.u(off, self.sl)

    def at(self, rel: int) -> int:
        """File offset of an HDF5 address."""
        return self.base + rel

    def _find_superblock(self) -> int:
        off = 0
        while off + 8 <= len(self.d):
            if self.d[off:off + 8] == SIGNATURE:
                return off
            off = 512 if off == 0 else off * 2
        raise H5Error("no HDF5 superblock (not a MATLAB v7.3 file)")

    def _superblock(self) -> None:
        p = self.sb + 8
        ver = self.d[p]
        self.sb_version = ver
        if ver in (0, 1):
            self.so, self.sl = self.d[p + 5], self.d[p + 6]
            q = p + 8 + 4 + 4  # leaf K, internal K, consistency flags
            if ver == 1:
                q += 4  # indexed-storage internal K + reserved
            base = self.addr(q)
            self.base = base if base else self.sb
            q += 4 * self.so  # base, free-space info, end of file, driver info
            # root group symbol-table entry: link name offset, object header address, ...
            self.root = self.addr(q + self.so)
        elif ver in (2, 3):
            self.so, self.sl = self.d[p + 1], self.d[p + 2]
            q = p + 4
            base = self.addr(q)
            self.base = base if base else self.sb
            q += 2 * self.so  # base, superblock extension
            q += self.so      # end of file
            self.root = self.addr(q)
        else:
            raise H5Error(f"superblock version {ver} is not supported")

    # -- object headers -------------------------------------------------------
    def messages(self, rel: int):
        """[(type, data_offset, size)] of the object header at address rel."""
        off = self.at(rel)
        out = []
        if self.d[off:off + 4] == b"OHDR":
            ver, flags = self.d[off + 4], self.d[off + 5]
            if ver != 2:
                raise H5Error(f"object header version {ver}")
            p = off + 6
            if flags & 0x20:
                p += 16
            if flags & 0x10:
                p += 4
            nsz = 1 << (flags & 3)
            size0 = self.u(p, nsz)
            p += nsz
            blocks = [(p, size0)]
            track_order = bool(flags & 0x04)
            while blocks:
                start, size = blocks.pop(0)
                q, end = start, start + size
                while q + 4 <= end:
                    mtype, msize, mflags = self.d[q], self.u(q + 1, 2), self.d[q + 3]
                    q += 4 + (2 if track_order else 0)
                    if mtype == 0x10:  # continuation
                        c_off, c_len = self.addr(q), self.length(q + self.so)
                        cs = self.at(c_off)
                        if self.d[cs:cs + 4] != b"OCHK":
                            raise H5Error("bad continuation block")
                        blocks.append((cs + 4, c_len - 8))
                    elif mtype != 0:
                        out.append((mtype, q, msize, mflags))
                    q += msize
            return out
        ver = self.d[off]
        if ver != 1:
            raise H5Error(f"object header version {ver} at {off}")
        nmsg, hsize = self.u(off + 2, 2), self.u(off + 8, 4)
        blocks = [(off + 16, hsize)]
        seen = 0
        while blocks and seen < nmsg:
            start, size = blocks.pop(0)
            q, end = start, start + size
            while q + 8 <= end and seen < nmsg:
                mtype, msize, mflags = self.u(q, 2), self.u(q + 2, 2), self.d[q + 4]
                q += 8
                seen += 1
                if mtype == 0x10:
                    blocks.append((self.at(self.addr(q)), self.length(q + self.so)))
                elif mtype != 0:
                    out.append((mtype, q, msize, mflags))
                q += msize
        return out

    # -- groups ---------------------------------------------------------------
    def children(self, rel: int):
        """{name: object header address} of a group, or None if not a group."""
        msgs = self.messages(rel)
        links = {}
        is_group = False
        for mtype, q, size, _ in msgs:
            if mtype == 0x11:  # symbol table: v1 B-tree + local heap
                is_group = True
                btree, heap = self.addr(q), self.addr(q + self.so)
                links.update(self._symbol_table(btree, heap))
            elif mtype == 0x06:  # link message (compact new-style group)
                is_group = True
                name, target = self._link(q)
                if target is not None:
                    links[name] = target
            elif mtype == 0x02:  # link info
                is_group = True
                heap_addr = self.addr(q + 2 + (8 if self.d[q + 1] & 1 else 0))
                if heap_addr != UNDEF:
                    raise NotImplementedError("group with dense link storage (fractal heap)")
        return links if is_group else None

    def _local_heap_data(self, heap: int) -> int:
        h = self.at(heap)
        if self.d[h:h + 4] != b"HEAP":
            raise H5Error("bad local heap")
        return self.at(self.addr(h + 8 + 2 * self.sl))

    def _nul(self, off: int) -> int:
        end = self.d.find(b"\x00", off)
        if end < 0:
            raise H5Error(f"unterminated string at {off}")
        return end

    def _cstr(self, off: int) -> str:
        end = self._nul(off)
        return self.d[off:end].decode("utf-8", "replace")

    def _symbol_table(self, btree: int, heap: int):
        names = {}
        hdata = self._local_heap_data(heap)

        def node(rel):
            n = self.at(rel)
            if self.d[n:n + 4] == b"TREE":
                if self.d[n + 4] != 0:
                    raise H5Error("group B-tree of the wrong type")
                level, used = self.d[n + 5], self.u(n + 6, 2)
                p = n + 8 + 2 * self.so + self.sl  # siblings, key 0
                for _ in range(used):
                    child = self.addr(p)
                    node(child) if level > 0 else snod(child)
                    p += self.so + self.sl
            else:
                snod(rel)

        def snod(rel):
            s = self.at(rel)
            if self.d[s:s + 4] != b"SNOD":
                raise H5Error("bad symbol node")
            count = self.u(s + 6, 2)
            p = s + 8
            esz = 2 * self.so + 24
            for _ in range(count):
                name = self._cstr(hdata + self.addr(p))
                names[name] = self.addr(p + self.so)
                p += esz

        node(btree)
        return names

    def _link(self, q: int):
        flags = self.d[q + 1]
        p = q + 2
        ltype = 0
        if flags & 0x08:
            ltype = self.d[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        nlen_sz = 1 << (flags & 3)
        nlen = self.u(p, nlen_sz)
        p += nlen_sz
        name = self.d[p:p + nlen].decode("utf-8", "replace")
        p += nlen
        return name, (self.addr(p) if ltype == 0 else None)

    # -- datatypes, dataspaces ------------------------------------------------
    def dtype(self, q: int):
        """(numpy dtype or ('string', n), encoded size) of the datatype at q."""
        cv = self.d[q]
        cls, ver = cv & 0x0F, cv >> 4
        bits = self.u(q + 1, 3)
        size = self.u(q + 4, 4)
        p = q + 8
        if cls == 0:  # fixed point
            order = ">" if bits & 1 else "<"
            kind = "i" if bits & 0x08 else "u"
            return np.dtype(f"{order}{kind}{size}"), 8 + 4
        if cls == 1:  # floating point
            if bits & 0x40:
                raise NotImplementedError("VAX floating-point order")
            order = ">" if bits & 1 else "<"
            return np.dtype(f"{order}f{size}"), 8 + 12
        if cls == 3:  # fixed-length string
            return ("string", size), 8
        if cls == 6:  # compound
            nmemb = bits & 0xFFFF
            names, formats, offsets = [], [], []
            for _ in range(nmemb):
                end = self._nul(p)
                name = self.d[p:end].decode("ascii", "replace")
                if ver < 3:
                    p += ((end - p) // 8 + 1) * 8  # null-terminated, padded to 8
                    moff = self.u(p, 4)
                    p += 4
                    if ver == 1:
                        p += 28  # dimensionality, reserved, permutation, reserved, dims
                else:
                    p = end + 1
                    nb = max(1, (size.bit_length() + 7) // 8)
                    moff = self.u(p, nb)
                    p += nb
                mdt, msz = self.dtype(p)
                p += msz
                if not isinstance(mdt, np.dtype):
                    raise NotImplementedError("compound member of a non-numeric type")
                names.append(name)
                formats.append(mdt)
                offsets.append(moff)
            return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size}), p - q
        raise NotImplementedError(f"HDF5 datatype class {cls} (MATLAB cell, reference or string data)")

    def dataspace(self, q: int):
        ver, rank, flags = self.d[q], self.d[q + 1], self.d[q + 2]
        p = q + (8 if ver == 1 else 4)
        if ver == 2 and self.d[q + 3] == 2:  # null dataspace
            return None
        return tuple(self.length(p + i * self.sl) for i in range(rank))

    # -- data -----------------------------------------------------------------
    def _filters(self, q: int):
        ver, n = self.d[q], self.d[q + 1]
        p = q + (8 if ver == 1 else 2)
        out = []
        for _ in range(n):
            fid = self.u(p, 2)
            if ver == 1 or fid >= 256:
                nlen = self.u(p + 2, 2)
                p += 4
            else:
                nlen = 0
                p += 2
            nval = self.u(p + 2, 2)
            p += 4
            if ver == 1:
                p += ((nlen + 7) // 8) * 8
            else:
                p += nlen
            vals = [self.u(p + 4 * i, 4) for i in range(nval)]
            p += 4 * nval
            if ver == 1 and nval % 2:
                p += 4
            out.append((fid, vals))
        return out

    def _unfilter(self, raw: bytes, filters, mask: int, itemsize: int) -> bytes:
        for i, (fid, vals) in reversed(list(enumerate(filters))):
            if mask & (1 << i):
                continue
            if fid == 1:  # deflate
                raw = zlib.decompress(raw)
            elif fid == 2:  # shuffle
                n = len(raw) // itemsize
                b = np.frombuffer(raw[:n * itemsize], np.uint8).reshape(itemsize, n)
                raw = b.T.tobytes() + raw[n * itemsize:]
            elif fid == 3:  # fletcher32 checksum: drop it
                raw = raw[:-4]
            else:
                raise NotImplementedError(f"HDF5 filter {fid}")
        return raw

    def read_dataset(self, msgs):
        shape = dt = layout = None
        filters = []
        for mtype, q, size, _ in msgs:
            if mtype == 0x01:
                shape = self.dataspace(q)
            elif mtype == 0x03:
                dt, _ = self.dtype(q)
            elif mtype == 0x08:
                layout = q
            elif mtype == 0x0B:
                filters = self._filters(q)
        if dt is None or layout is None:
            raise H5Error("dataset without datatype or layout")
        if shape is None:
            return None
        if not isinstance(dt, np.dtype):
            raise NotImplementedError("string-valued dataset")
        n = int(np.prod(shape)) if shape else 1
        nbytes = n * dt.itemsize
        ver = self.d[layout]
        if ver in (1, 2):
            # version, dimensionality, class, 5 reserved, [address], dimension sizes (4 bytes)
            ndim, lclass = self.d[layout + 1], self.d[layout + 2]
            p = layout + 8
            a = UNDEF
            if lclass != 0:
                a = self.addr(p)
                p += self.so
            dims = [self.u(p + 4 * i, 4) for i in range(ndim)]
            p += 4 * ndim
            if lclass == 0:
                sz = self.u(p, 4)
                raw = self.d[p + 4:p + 4 + sz]
            elif lclass == 1:
                raw = b"\x00" * nbytes if a == UNDEF else self.d[self.at(a):self.at(a) + nbytes]
            elif lclass == 2:
                out = np.zeros(shape, dt)
                if a != UNDEF:
                    self._chunks(a, ndim - 1, dims[:ndim - 1], shape, dt, filters, out)
                return out
            else:
                raise NotImplementedError(f"data layout class {lclass}")
        elif ver == 3:
            lclass = self.d[layout + 1]
            if lclass == 0:  # compact
                sz = self.u(layout + 2, 2)
                raw = self.d[layout + 4:layout + 4 + sz]
            elif lclass == 1:  # contiguous
                a = self.addr(layout + 2)
                raw = b"\x00" * nbytes if a == UNDEF else self.d[self.at(a):self.at(a) + nbytes]
            elif lclass == 2:  # chunked, v1 B-tree
                rank = self.d[layout + 2] - 1
                bt = self.addr(layout + 3)
                cdims = [self.u(layout + 3 + self.so + 4 * i, 4) for i in range(rank)]
                out = np.zeros(shape, dt)
                if bt != UNDEF:
                    self._chunks(bt, rank, cdims, shape, dt, filters, out)
                return out
            else:
                raise NotImplementedError(f"data layout class {lclass}")
        else:
            raise NotImplementedError(f"data layout message version {ver}")
        if len(raw) < nbytes:
            raise H5Error("dataset shorter than its dataspace")
        return np.frombuffer(raw[:nbytes], dt).reshape(shape).copy()

    def _chunks(self, rel, rank, cdims, shape, dt, filters, out):
        n = self.at(rel)
        if self.d[n:n + 4] != b"TREE" or self.d[n + 4] != 1:
            raise H5Error("bad chunk B-tree")
        level, used = self.d[n + 5], self.u(n + 6, 2)
        ksz = 8 + 8 * (rank + 1)
        p = n + 8 + 2 * self.so
        for _ in range(used):
            csize, mask = self.u(p, 4), self.u(p + 4, 4)
            offs = [self.u(p + 8 + 8 * i, 8) for i in range(rank)]
            child = self.addr(p + ksz)
            if level > 0:
                self._chunks(child, rank, cdims, shape, dt, filters, out)
            else:
                c = self.at(child)
                raw = self._unfilter(self.d[c:c + csize], filters, mask, dt.itemsize)
                block = np.frombuffer(raw[:int(np.prod(cdims)) * dt.itemsize], dt).reshape(cdims)
                sl_out = tuple(slice(o, min(o + cd, s)) for o, cd, s in zip(offs, cdims, shape))
                sl_in = tuple(slice(0, s.stop - s.start) for s in sl_out)
                out[sl_out] = block[sl_in]
            p += ksz + self.so

    def attributes(self, msgs):
        out = {}
        for mtype, q, size, _ in msgs:
            if mtype != 0x0C:
                continue
            ver = self.d[q]
            nsz, tsz, ssz = self.u(q + 2, 2), self.u(q + 4, 2), self.u(q + 6, 2)
            p = q + 8 + (1 if ver == 3 else 0)
            pad = (lambda x: (x + 7) // 8 * 8) if ver == 1 else (lambda x: x)
            name = self.d[p:p + nsz].split(b"\x00")[0].decode("ascii", "replace")
            p += pad(nsz)
            dt, _ = self.dtype(p)
            p += pad(tsz)
            shape = self.dataspace(p)
            p += pad(ssz)
            if isinstance(dt, tuple):  # string
                out[name] = self.d[p:p + dt[1]].split(b"\x00")[0].decode("ascii", "replace")
            elif shape is not None:
                cnt = int(np.prod(shape)) if shape else 1
                v = np.frombuffer(self.d[p:p + cnt * dt.itemsize], dt)
                out[name] = v.reshape(shape) if shape else v[0]
        return out


def _transpose(arr):
    """MATLAB is column-major: an [a, b, c] array is stored as HDF5 [c, b, a]
    (utils/io.py:_transpose)."""
    return np.transpose(arr) if arr.ndim >= 2 else arr


def _to_numpy(f: _File, msgs):
    raw = f.read_dataset(msgs)
    if raw is None:
        return np.zeros((0,))
    if raw.dtype.fields and {"real", "imag"} <= set(raw.dtype.fields):
        return _transpose(np.array(raw["real"]) + 1j * np.array(raw["imag"]))
    attrs = f.attributes(msgs)
    mc = attrs.get("MATLAB_complex", 0)
    if np.ndim(mc) and np.size(mc):
        mc = np.ravel(mc)[0]
    if mc:
        arr = np.array(raw)
        if arr.shape[0] == 2:
            return _transpose(arr[0] + 1j * arr[1])
        if arr.shape[-1] == 2:
            return _transpose(arr[..., 0] + 1j * arr[..., 1])
    return _transpose(np.array(raw))


def _convert(f: _File, rel: int, depth: int = 0):
    if depth > 32:
        raise H5Error("group nesting too deep")
    kids = f.children(rel)
    if kids is None:
        return _to_numpy(f, f.messages(rel))
    if "real" in kids and "imag" in kids:
        return _convert(f, kids["real"], depth + 1) + 1j * _convert(f, kids["imag"], depth + 1)
    return {k: _convert(f, v, depth + 1) for k, v in kids.items() if not k.startswith("#")}


def is_hdf5(path: str) -> bool:
    with open(path, "rb") as fh:
        head = fh.read(4096 + 8)
    return any(head[o:o + 8] == SIGNATURE for o in (0, 512, 1024, 2048, 4096))


def read_mat73(path: str, key: str | None = None) -> dict:
    """Variables of a MATLAB v7.3 file (utils/io.py:read_data, h5py branch).
    The file is memory-mapped: only the pages of the objects read are loaded."""
    with open(path, "rb") as fh:
        size = fh.seek(0, 2)
        if size == 0:
            raise H5Error("empty file")
        with mmap.mmap(fh.fileno(), 0, access=mmap.ACCESS_READ) as mm:
            f = _File(mm)
            top = f.children(f.root)
            if top is None:
                raise H5Error("the root object is not a group")
            if key and key in top:
                return {key: _convert(f, top[key])}
            return {k: _convert(f, v) for k, v in top.items() if not k.startswith("#")}
