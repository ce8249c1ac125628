"""A minimal HDF5 writer for test meshes (test infrastructure only).

Writes a mesh dict (the oracle's format) in the layout the reference's
MeshHDF5Source reads (MeshHDF5Source.cpp: root attributes ncel, nfac, nbnd,
nreg; /cell, /face, /bnd, /reg groups; 1-based labels; cell2 = 0 on boundary
faces), in the oldest HDF5 structures as the HDF Group's File Format
Specification describes them: superblock version 0, groups in symbol tables
(one version 1 B-tree group node, one symbol table node, a local heap),
version 1 object headers, version 1 dataspaces, little-endian int32 and
float64 datatypes, version 3 contiguous layouts, version 1 attributes.
Only what the library's reader needs; nothing here is used by the library.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K, NODE_K = 4, 16


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


def _dtype(arr):
    if arr.dtype.kind in "iu":
        return bytes([0x10, 0x08, 0, 0]) + struct.pack("<I", 4) + struct.pack("<HH", 0, 32), "<i4"
    props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
    return bytes([0x11, 0x20, 63, 0]) + struct.pack("<I", 8) + props, "<f8"


def _space(shape):
    return bytes([1, len(shape), 0, 0]) + b"\0" * 4 + b"".join(struct.pack("<Q", int(n)) for n in shape)


def _msg(mtype, body):
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), 0) + body


class _File:
    def __init__(self):
        self.buf = bytearray(96)  # superblock + root symbol table entry, filled in last

    def alloc(self, data: bytes) -> int:
        addr = len(self.buf)
        self.buf += _pad8(data)
        return addr

    def object_header(self, msgs) -> int:
        body = b"".join(msgs)
        head = struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\0" * 4
        return self.alloc(head + body)

    def dataset(self, arr) -> int:
        arr = np.ascontiguousarray(arr)
        dt, code = _dtype(arr)
        raw = arr.astype(code).tobytes()
        data = self.alloc(raw)
        layout = bytes([3, 1]) + struct.pack("<QQ", data, len(raw))
        return self.object_header([_msg(0x01, _space(arr.shape)), _msg(0x03, dt), _msg(0x08, layout)])

    def group(self, entries, attrs=()):
        """entries: {name: object header address}; returns (header, btree, heap)."""
        names = sorted(entries)
        assert len(names) <= 2 * LEAF_K, "one symbol table node per group"
        heap_data = bytearray(b"\0" * 8)   # offset 0: the empty name
        offs = {}
        for n in names:
            offs[n] = len(heap_data)
            heap_data += _pad8(n.encode() + b"\0")
        heap_data_addr = self.alloc(bytes(heap_data))
        heap = self.alloc(b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap_data), UNDEF, heap_data_addr))
        snod = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(names)))
        for n in names:
            snod += struct.pack("<QQI4x", offs[n], entries[n], 0) + b"\0" * 16
        snod += b"\0" * (40 * (2 * LEAF_K - len(names)))
        snod_addr = self.alloc(bytes(snod))
        tree = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", 1, UNDEF, UNDEF))
        tree += struct.pack("<QQQ", 0, snod_addr, offs[names[-1]] if names else 0)
        tree += b"\0" * (8 * (2 * NODE_K + 1) + 8 * 2 * NODE_K - 24)
        btree = self.alloc(bytes(tree))
        msgs = [_msg(0x11, struct.pack("<QQ", btree, heap))]
        for name, value in attrs:
            nm = name.encode() + b"\0"
            dt, _ = _dtype(np.zeros(1, np.int32))
            sp = _space((1,))
            body = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(sp)) + _pad8(nm) + _pad8(dt) + _pad8(sp)
            msgs.append(_msg(0x0C, body + struct.pack("<i", int(value))))
        return self.object_header(msgs), btree, heap

    def finish(self, root_header, root_btree, root_heap) -> bytes:
        sb = b"\x89HDF\r\n\x1a\n" + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", LEAF_K, NODE_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, len(self.buf), UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, root_header, 1, root_btree, root_heap)
        assert len(sb) == 96
        self.buf[:96] = sb
        return bytes(self.buf)


def mesh_hdf5_bytes(m, bnd_distance=None) -> bytes:
    """HDF5 file bytes of mesh ``m`` (oracle dict with regions)."""
    nC, nF, nB = int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"])
    nR = int(m.get("nRegions", 1))
    f = _File()
    c2 = np.asarray(m["faceCell2"])
    fb = np.asarray(m["faceBnd"])
    face = {
        "cell1": f.dataset(np.asarray(m["faceCell1"], np.int32) + 1),
        "cell2": f.dataset(np.where(c2 >= 0, c2 + 1, 0).astype(np.int32)),
        "bnd": f.dataset(np.where(fb >= 0, fb + 1, 0).astype(np.int32)),
        "lambda": f.dataset(np.asarray(m["faceLambda"], np.float64)),
        "area": f.dataset(np.asarray(m["faceArea"], np.float64)),
        "n": f.dataset(np.asarray(m["faceNorm"], np.float64).reshape(nF, 3)),
        "x": f.dataset(np.asarray(m["faceCenter"], np.float64).reshape(nF, 3)),
    }
    cell = {"x": f.dataset(np.asarray(m["cellCenter"], np.float64).reshape(nC, 3)),
            "vol": f.dataset(np.asarray(m["cellVolume"], np.float64))}
    dist = np.zeros(nB) if bnd_distance is None else np.asarray(bnd_distance, np.float64)
    bnd = {"rid": f.dataset(np.asarray(m.get("bndRegion", np.zeros(nB, np.int32)), np.int32) + 1),
           "distance": f.dataset(dist)}
    groups = {}
    for gname, ents in (("cell", cell), ("face", face), ("bnd", bnd)):
        groups[gname] = f.group(ents)[0]
    root = f.group(groups, attrs=(("ncel", nC), ("nfac", nF), ("nbnd", nB), ("nreg", nR)))
    return f.finish(*root)
