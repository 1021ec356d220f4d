"""Minimal HDF5 writer for test fixtures (test infrastructure only).

Writes the subset that TRIQS h5 produces for flat groups and that ``coqui_b200.h5lite``
reads: superblock version 0, one root group (version-1 object header, symbol-table message,
v1 B-tree with one symbol node, local heap), and datasets with version-1 object headers
(dataspace v1, IEEE little-endian float or signed integer datatype, contiguous layout v3).
Complex arrays are written as TRIQS does, with a trailing (re, im) dimension.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


def _pad8(b: bytes) -> bytes:
    return b + b"\x00" * (-len(b) % 8)


def _msg(mtype: int, body: bytes) -> bytes:
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), 0) + body


def _object_header(messages) -> bytes:
    data = b"".join(messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(data)) + data


def _dataspace(shape) -> bytes:
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", n) for n in shape)


def _datatype(dt: np.dtype) -> bytes:
    if dt.kind == "f":
        return (struct.pack("<BBBBI", (1 << 4) | 1, 0x20, dt.itemsize * 8 - 1, 0, dt.itemsize)
                + struct.pack("<HHBBBBI", 0, dt.itemsize * 8, 52, 11, 0, 52, 1023))
    if dt.kind == "i":
        return (struct.pack("<BBBBI", (1 << 4) | 0, 0x08, 0, 0, dt.itemsize)
                + struct.pack("<HH", 0, dt.itemsize * 8))
    raise ValueError(f"dtype {dt} not supported")


def write_h5(path: str, datasets: dict) -> None:
    """Write {name: array} as datasets of the root group (complex -> trailing (re, im))."""
    items = []
    for name in sorted(datasets):
        a = np.asarray(datasets[name])
        if np.iscomplexobj(a):
            a = np.stack([a.real, a.imag], axis=-1).astype(np.float64)
        elif a.dtype.kind == "f":
            a = a.astype("<f8")
        elif a.dtype.kind in "iub":
            a = a.astype("<i8" if a.dtype.itemsize > 4 else "<i4")
        items.append((name, np.ascontiguousarray(a)))
    buf = bytearray(96)  # superblock, filled at the end

    def place(b: bytes) -> int:
        while len(buf) % 8:
            buf.append(0)
        addr = len(buf)
        buf.extend(b)
        return addr

    # local heap: "" at offset 0, then the names
    heap_data = bytearray(8)
    name_off = {}
    for name, _ in items:
        name_off[name] = len(heap_data)
        heap_data.extend(_pad8(name.encode() + b"\x00"))
    heap_data_addr = place(bytes(heap_data))
    heap_addr = place(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), UNDEF, heap_data_addr))
    # datasets
    headers = {}
    for name, a in items:
        data_addr = place(a.tobytes())
        layout = struct.pack("<BBQQ", 3, 1, data_addr, a.nbytes)
        headers[name] = place(_object_header([_msg(0x01, _dataspace(a.shape)),
                                              _msg(0x03, _datatype(a.dtype)),
                                              _msg(0x08, layout)]))
    # one symbol node with every entry (names sorted), one B-tree leaf pointing at it
    snod = b"SNOD" + struct.pack("<BBH", 1, 0, len(items))
    for name, _ in items:
        snod += struct.pack("<QQI4x16x", name_off[name], headers[name], 0)
    snod_addr = place(snod)
    last = name_off[items[-1][0]] if items else 0
    tree_addr = place(b"TREE" + struct.pack("<BBHQQ", 0, 0, 1, UNDEF, UNDEF)
                      + struct.pack("<QQQ", 0, snod_addr, last))
    root = place(_object_header([_msg(0x11, struct.pack("<QQ", tree_addr, heap_addr))]))
    eof = len(buf)
    sb = b"\x89HDF\r\n\x1a\n" + struct.pack("<BBBBBBBB", 0, 0, 0, 0, 0, 8, 8, 0)
    sb += struct.pack("<HHI", 32, 16, 0)  # leaf K (room for 64 symbols per node), internal K
    sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    sb += struct.pack("<QQII", 0, root, 1, 0) + struct.pack("<QQ", tree_addr, heap_addr)
    assert len(sb) == 96
    buf[:96] = sb
    with open(path, "wb") as f:
        f.write(bytes(buf))
