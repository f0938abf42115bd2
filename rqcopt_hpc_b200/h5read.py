"""Minimal read-only HDF5 reader for the files of the rqcopt_hpc project: the test
fixtures (test/data/*.hdf5) and the example inputs and outputs (examples/*/*.hdf5).

Those files are small HDF5 files written by h5py or libhdf5 with the "earliest" file
format: superblock version 0, a root group stored as a symbol table (version-1 B-tree
plus local heap), version-1 object headers, and contiguous or compact datasets of
little-endian IEEE doubles or integers.  Only that subset is implemented; anything
else raises ``ValueError``.  It exists because h5py and libhdf5 are not available
everywhere this library runs.

    from rqcopt_hpc_b200 import h5read
    arrays = h5read.read_all("ising1d_dynamics_opt_n3_init.hdf5")   # {name: numpy array}
"""
from __future__ import annotations

import struct

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"


class H5File:
    def __init__(self, path: str):
        with open(path, "rb") as fh:
            self.buf = fh.read()
        if self.buf[:8] != _SIG:
            raise ValueError(f"{path}: not an HDF5 file")
        if self.buf[8] != 0:
            raise ValueError(f"{path}: superblock version {self.buf[8]} not supported")
        self.so = self.buf[13]  # size of offsets
        self.sl = self.buf[14]  # size of lengths
        if self.so != 8 or self.sl != 8:
            raise ValueError("only 8-byte offsets and lengths are supported")
        # root group symbol table entry starts at byte 56
        ent = 56
        cache_type = self._u32(ent + 16)
        if cache_type != 1:
            raise ValueError("root group has no cached symbol table")
        btree = self._u64(ent + 24)
        heap = self._u64(ent + 32)
        self.datasets = {}
        for name, ohdr in self._group_entries(btree, heap):
            self.datasets[name] = ohdr

    # -- primitive reads
    def _u8(self, o):
        return self.buf[o]

    def _u16(self, o):
        return struct.unpack_from("<H", self.buf, o)[0]

    def _u32(self, o):
        return struct.unpack_from("<I", self.buf, o)[0]

    def _u64(self, o):
        return struct.unpack_from("<Q", self.buf, o)[0]

    # -- groups
    def _heap_name(self, heap, off):
        if self.buf[heap:heap + 4] != b"HEAP":
            raise ValueError("bad local heap signature")
        data = self._u64(heap + 24)
        start = data + off
        end = self.buf.index(b"\x00", start)
        return self.buf[start:end].decode()

    def _group_entries(self, node, heap):
        if self.buf[node:node + 4] != b"TREE":
            raise ValueError("bad B-tree signature")
        level = self._u8(node + 5)
        used = self._u16(node + 6)
        p = node + 8 + 16  # skip left/right sibling addresses
        p += self.sl  # key 0
        for _ in range(used):
            child = self._u64(p)
            p += self.so + self.sl
            if level > 0:
                yield from self._group_entries(child, heap)
            else:
                yield from self._snod(child, heap)

    def _snod(self, addr, heap):
        if self.buf[addr:addr + 4] != b"SNOD":
            raise ValueError("bad symbol-table node signature")
        n = self._u16(addr + 6)
        p = addr + 8
        for _ in range(n):
            name_off = self._u64(p)
            ohdr = self._u64(p + 8)
            yield self._heap_name(heap, name_off), ohdr
            p += 40

    # -- object headers
    def _messages(self, ohdr):
        if self._u8(ohdr) != 1:
            raise ValueError("only version-1 object headers are supported")
        nmsg = self._u16(ohdr + 2)
        size = self._u32(ohdr + 8)
        blocks = [(ohdr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p = start
            while p + 8 <= start + length and len(out) < nmsg:
                mtype = self._u16(p)
                msize = self._u16(p + 2)
                body = p + 8
                if mtype == 0x10:  # continuation
                    blocks.append((self._u64(body), self._u64(body + 8)))
                out.append((mtype, body, msize))
                p = body + msize
        return out

    def read(self, name: str) -> np.ndarray:
        ohdr = self.datasets[name]
        shape = dtype = layout = None
        for mtype, body, msize in self._messages(ohdr):
            if mtype == 0x01:
                shape = self._dataspace(body)
            elif mtype == 0x03:
                dtype = self._datatype(body)
            elif mtype == 0x08:
                layout = (body, msize)
        if shape is None or dtype is None or layout is None:
            raise ValueError(f"{name}: missing dataspace, datatype or layout message")
        raw = self._layout_bytes(*layout, nbytes=int(np.prod(shape, dtype=np.int64)) * dtype.itemsize)
        return np.frombuffer(raw, dtype=dtype).reshape(shape).copy()

    def _dataspace(self, b):
        version = self._u8(b)
        ndims = self._u8(b + 1)
        if version == 1:
            p = b + 8
        elif version == 2:
            p = b + 4
        else:
            raise ValueError(f"dataspace version {version} not supported")
        return tuple(self._u64(p + 8 * k) for k in range(ndims))

    def _datatype(self, b):
        cls = self._u8(b) & 0x0F
        bits0 = self._u8(b + 1)
        size = self._u32(b + 4)
        if bits0 & 1:
            raise ValueError("big-endian data not supported")
        if cls == 0:
            signed = bool(bits0 & 0x08)
            return np.dtype(f"<{'i' if signed else 'u'}{size}")
        if cls == 1:
            return np.dtype(f"<f{size}")
        raise ValueError(f"datatype class {cls} not supported")

    def _layout_bytes(self, b, msize, nbytes):
        version = self._u8(b)
        if version == 3:
            cls = self._u8(b + 1)
            if cls == 0:  # compact
                size = self._u16(b + 2)
                return self.buf[b + 4:b + 4 + size][:nbytes]
            if cls == 1:  # contiguous
                addr = self._u64(b + 2)
                return self.buf[addr:addr + nbytes]
            raise ValueError("chunked datasets are not supported")
        if version in (1, 2):
            ndims = self._u8(b + 1)
            cls = self._u8(b + 2)
            if cls == 1:
                addr = self._u64(b + 8)
                return self.buf[addr:addr + nbytes]
            if cls == 0:
                p = b + 8 + 4 * ndims
                size = self._u32(p)
                return self.buf[p + 4:p + 4 + size][:nbytes]
            raise ValueError("chunked datasets are not supported")
        raise ValueError(f"layout version {version} not supported")


def read_all(path: str) -> dict:
    f = H5File(path)
    return {name: f.read(name) for name in sorted(f.datasets)}
