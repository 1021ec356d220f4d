"""Minimal read-only HDF5 decoder for the IR sparse-sampling tables.

The imaginary-axis tables that CoQui ships (``src/numerics/imag_axes_ft/ir/data/*.h5``,
written by ``gen_sparse_ir.py`` through TRIQS h5) and its Green's-function test fixtures
use a small subset of HDF5:

* superblock version 0 with 8-byte offsets and lengths,
* version-1 object headers with continuation blocks,
* old-style groups (symbol-table message -> v1 B-tree of SNOD nodes + local heap),
* contiguous, compact or chunked datasets, chunked ones optionally deflate-compressed
  (filter 1) and byte-shuffled (filter 2),
* little-endian integer / IEEE float element types; complex values are stored by
  TRIQS h5 as a trailing dimension of length 2 (re, im).

Only that subset is decoded.  The decoder is pure Python (``struct``, ``zlib``, numpy),
because h5py is not available where the tables are converted.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"


class H5Error(RuntimeError):
    pass


class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        if data[:8] != _SIG:
            raise H5Error("not an HDF5 file")
        ver = data[8]
        if ver not in (0, 1):
            raise H5Error(f"unsupported superblock version {ver}")
        self.so = data[13]
        self.sl = data[14]
        if self.so != 8 or self.sl != 8:
            raise H5Error("only 8-byte offsets/lengths supported")
        p = 24 + (4 if ver == 1 else 0)
        self.base = self.u64(p)
        p += 4 * 8  # base, free-space, eof, driver
        # root group symbol table entry
        self.root_header = self.u64(p + 8)

    # -- primitive readers ---------------------------------------------------------
    def u8(self, p):
        return self.d[p]

    def u16(self, p):
        return struct.unpack_from("<H", self.d, p)[0]

    def u32(self, p):
        return struct.unpack_from("<I", self.d, p)[0]

    def u64(self, p):
        return struct.unpack_from("<Q", self.d, p)[0]

    # -- object headers ------------------------------------------------------------
    def messages(self, addr):
        """Yield (type, body_offset, size) for every message of a v1 object header."""
        if self.u8(addr) != 1:
            raise H5Error(f"unsupported object header version {self.u8(addr)} at {addr}")
        nmsg = self.u16(addr + 2)
        hsize = self.u32(addr + 8)
        blocks = [(addr + 16, hsize)]
        out = []
        while blocks and len(out) < nmsg:
            start, size = blocks.pop(0)
            p = start
            end = start + size
            while p + 8 <= end and len(out) < nmsg:
                mtype = self.u16(p)
                msize = self.u16(p + 2)
                body = p + 8
                out.append((mtype, body, msize))
                if mtype == 0x10:  # continuation
                    blocks.append((self.u64(body), self.u64(body + 8)))
                p = body + msize
        return out

    # -- groups --------------------------------------------------------------------
    def _heap_data(self, heap_addr):
        if self.d[heap_addr:heap_addr + 4] != b"HEAP":
            raise H5Error("bad local heap")
        return self.u64(heap_addr + 24)

    def _cstr(self, p):
        e = self.d.index(b"\x00", p)
        return self.d[p:e].decode()

    def _btree_group(self, node, heap_data, out):
        if self.d[node:node + 4] != b"TREE":
            raise H5Error("bad group B-tree node")
        ntype, level, used = self.u8(node + 4), self.u8(node + 5), self.u16(node + 6)
        if ntype != 0:
            raise H5Error("expected group B-tree")
        p = node + 24 + 8  # skip siblings, then key0
        for _ in range(used):
            child = self.u64(p)
            p += 16  # child + next key
            if level > 0:
                self._btree_group(child, heap_data, out)
            else:
                self._snod(child, heap_data, out)

    def _snod(self, addr, heap_data, out):
        if self.d[addr:addr + 4] != b"SNOD":
            raise H5Error("bad symbol table node")
        n = self.u16(addr + 6)
        p = addr + 8
        for _ in range(n):
            name = self._cstr(heap_data + self.u64(p))
            out[name] = self.u64(p + 8)
            p += 40

    def children(self, header):
        for mtype, body, _ in self.messages(header):
            if mtype == 0x11:
                btree, heap = self.u64(body), self.u64(body + 8)
                out = {}
                self._btree_group(btree, self._heap_data(heap), out)
                return out
        return None

    # -- datasets ------------------------------------------------------------------
    def dataset(self, header):
        shape = dtype = layout = None
        filters = []
        for mtype, body, size in self.messages(header):
            if mtype == 0x01:
                shape = self._dataspace(body)
            elif mtype == 0x03:
                dtype = self._datatype(body)
            elif mtype == 0x08:
                layout = (body, size)
            elif mtype == 0x0B:
                filters = self._filters(body)
        if shape is None or dtype is None or layout is None:
            raise H5Error("object is not a dataset")
        if isinstance(dtype, str):
            return dtype  # variable-length string marker
        return self._read_layout(layout[0], shape, dtype, filters)

    def _dataspace(self, p):
        ver, ndim, flags = self.u8(p), self.u8(p + 1), self.u8(p + 2)
        if ver == 1:
            q = p + 8
        elif ver == 2:
            if self.u8(p + 3) == 0:  # scalar
                return ()
            q = p + 4
        else:
            raise H5Error(f"dataspace version {ver}")
        return tuple(self.u64(q + 8 * i) for i in range(ndim))

    def _datatype(self, p):
        cv = self.u8(p)
        cls = cv & 0x0F
        bits0 = self.u8(p + 1)
        size = self.u32(p + 4)
        if cls in (3, 9):
            return "string"
        if bits0 & 1:
            raise H5Error("big-endian data not supported")
        if cls == 0:
            signed = bool(bits0 & 0x08)
            return np.dtype(("<i" if signed else "<u") + str(size))
        if cls == 1:
            return np.dtype("<f" + str(size))
        raise H5Error(f"datatype class {cls} not supported")

    def _filters(self, p):
        ver, nf = self.u8(p), self.u8(p + 1)
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(nf):
            fid = self.u16(q)
            if ver == 1 or fid >= 256:
                nlen = self.u16(q + 2)
                flags, nval = self.u16(q + 4), self.u16(q + 6)
                q += 8
                if ver == 1:
                    nlen = (nlen + 7) & ~7
                q += nlen
            else:
                flags, nval = self.u16(q + 2), self.u16(q + 4)
                q += 6
            vals = [self.u32(q + 4 * i) for i in range(nval)]
            q += 4 * nval
            if ver == 1 and nval % 2:
                q += 4
            out.append((fid, vals))
        return out

    def _read_layout(self, p, shape, dtype, filters):
        ver = self.u8(p)
        count = int(np.prod(shape)) if shape else 1
        if ver == 3:
            cls = self.u8(p + 1)
            if cls == 0:
                n = self.u16(p + 2)
                raw = self.d[p + 4:p + 4 + n]
                return np.frombuffer(raw, dtype, count).reshape(shape)
            if cls == 1:
                addr = self.u64(p + 2)
                return np.frombuffer(self.d, dtype, count, addr).reshape(shape)
            if cls == 2:
                nd = self.u8(p + 2)
                btree = self.u64(p + 3)
                cdims = [self.u32(p + 11 + 4 * i) for i in range(nd)]
                return self._chunked(btree, shape, cdims[:-1], dtype, filters)
            raise H5Error(f"layout class {cls}")
        if ver in (1, 2):
            nd, cls = self.u8(p + 1), self.u8(p + 2)
            q = p + 8
            if cls == 0:
                dims = [self.u32(q + 4 * i) for i in range(nd)]
                q += 4 * nd
                n = self.u32(q)
                return np.frombuffer(self.d[q + 4:q + 4 + n], dtype, count).reshape(shape)
            addr = self.u64(q)
            q += 8
            dims = [self.u32(q + 4 * i) for i in range(nd)]
            if cls == 1:
                return np.frombuffer(self.d, dtype, count, addr).reshape(shape)
            return self._chunked(addr, shape, dims[:-1], dtype, filters)
        raise H5Error(f"layout version {ver}")

    def _chunked(self, btree, shape, cdims, dtype, filters):
        out = np.zeros(shape, dtype)
        rank = len(shape)
        chunks = []
        self._btree_chunks(btree, rank, chunks)
        csize = int(np.prod(cdims))
        for offs, nbytes, mask, addr in chunks:
            raw = self.d[addr:addr + nbytes]
            for i, (fid, vals) in reversed(list(enumerate(filters))):
                if mask & (1 << i):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    es = vals[0] if vals else dtype.itemsize
                    a = np.frombuffer(raw, np.uint8).reshape(es, -1)
                    raw = a.T.tobytes()
                else:
                    raise H5Error(f"filter {fid} not supported")
            block = np.frombuffer(raw, dtype, csize).reshape(cdims)
            sl_out = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
            sl_in = tuple(slice(0, x.stop - x.start) for x in sl_out)
            out[sl_out] = block[sl_in]
        return out

    def _btree_chunks(self, node, rank, out):
        if self.d[node:node + 4] != b"TREE":
            raise H5Error("bad chunk B-tree node")
        level, used = self.u8(node + 5), self.u16(node + 6)
        ksz = 8 + 8 * (rank + 1)
        p = node + 24
        for _ in range(used):
            nbytes, mask = self.u32(p), self.u32(p + 4)
            offs = [self.u64(p + 8 + 8 * i) for i in range(rank)]
            child = self.u64(p + ksz)
            if level > 0:
                self._btree_chunks(child, rank, out)
            else:
                out.append((offs, nbytes, mask, child))
            p += ksz + 8


def read_h5(path: str) -> dict:
    """Read every dataset of an HDF5 file into a nested dict of numpy arrays."""
    with open(path, "rb") as f:
        r = _Reader(f.read())

    def walk(header):
        kids = r.children(header)
        if kids is None:
            return r.dataset(header)
        return {name: walk(addr) for name, addr in kids.items()}

    return walk(r.root_header)


def as_complex(a: np.ndarray) -> np.ndarray:
    """TRIQS h5 stores complex arrays with a trailing (re, im) dimension."""
    a = np.asarray(a, dtype=np.float64)
    if a.shape[-1] != 2:
        raise H5Error("array has no trailing complex dimension")
    return a[..., 0] + 1j * a[..., 1]
