"""Minimal HDF5 reader for the tests: follows the published HDF5 file format
specification (superblock versions 0 and 1, version-1 object headers with
continuation blocks, symbol-table groups through a version-1 B-tree of group
nodes, symbol-table nodes and a local heap, contiguous and compact layouts,
fixed-point and IEEE floating-point datatypes).  Written independently of the
library's writer (cupf_b200/host/h5_writer.cpp) to check what it produces; no
libhdf5 or h5py exists in this environment.  Also reads files written by libhdf5
itself in that subset (tests/test_h5.py reads SciPy's MATLAB v7.3 test file).

    f = H5File(path); f.keys(); f[name] -> numpy array
"""
from __future__ import annotations

import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"


class H5FormatError(ValueError):
    pass


class H5File:
    def __init__(self, path):
        self.buf = open(path, "rb").read()
        self.base = self._find_superblock()
        self._parse_superblock()
        self._datasets = {}
        self._walk_group(self.root_btree, self.root_heap)

    # -- low-level helpers
    def _u(self, off, n):
        b = self.buf[off:off + n]
        if len(b) != n:
            raise H5FormatError("read past end of file at %d" % off)
        return int.from_bytes(b, "little")

    def _addr(self, off):
        v = self._u(off, self.so)
        return None if v == (1 << (8 * self.so)) - 1 else v

    def _abs(self, a):
        return self.base + a

    def _find_superblock(self):
        # the superblock is at 0 or at a power of two >= 512 (after a user block)
        off = 0
        while off < len(self.buf):
            if self.buf[off:off + 8] == SIGNATURE:
                return off
            off = 512 if off == 0 else off * 2
        raise H5FormatError("no HDF5 signature")

    def _parse_superblock(self):
        b = self.base
        ver = self.buf[b + 8]
        if ver not in (0, 1):
            raise H5FormatError("superblock version %d not supported" % ver)
        self.so = self.buf[b + 13]  # size of offsets
        self.sl = self.buf[b + 14]  # size of lengths
        self.leaf_k = self._u(b + 16, 2)
        self.internal_k = self._u(b + 18, 2)
        p = b + 24
        if ver == 1:
            p += 4  # indexed storage internal node K + reserved
        base_addr = self._u(p, self.so)
        # addresses are relative to the base address, which is the superblock's
        # own position when a user block precedes it
        self.base = base_addr if base_addr else b
        p += 4 * self.so  # base, free-space, end of file, driver info
        # root group symbol table entry
        self.root_header = self._addr(p + self.so)
        cache_type = self._u(p + 2 * self.so, 4)
        if cache_type == 1:
            scratch = p + 2 * self.so + 8
            self.root_btree = self._addr(scratch)
            self.root_heap = self._addr(scratch + self.so)
        else:
            msgs = self._object_messages(self.root_header)
            stab = [d for t, d in msgs if t == 0x11]
            if not stab:
                raise H5FormatError("root group has no symbol table message")
            self.root_btree = int.from_bytes(stab[0][:self.so], "little")
            self.root_heap = int.from_bytes(stab[0][self.so:2 * self.so], "little")

    # -- groups
    def _heap_data(self, heap_addr):
        a = self._abs(heap_addr)
        if self.buf[a:a + 4] != b"HEAP":
            raise H5FormatError("bad local heap signature")
        size = self._u(a + 8, self.sl)
        data_addr = self._u(a + 8 + 2 * self.sl, self.so)
        return self.buf[self._abs(data_addr):self._abs(data_addr) + size]

    @staticmethod
    def _cstr(heap, off):
        end = heap.index(b"\0", off)
        return heap[off:end].decode()

    def _walk_group(self, btree, heap_addr, prefix=""):
        heap = self._heap_data(heap_addr)
        for name, header in self._btree_entries(btree, heap):
            msgs = self._object_messages(header)
            types = [t for t, _ in msgs]
            if 0x11 in types:  # a subgroup
                d = dict(msgs)[0x11]
                self._walk_group(int.from_bytes(d[:self.so], "little"),
                                 int.from_bytes(d[self.so:2 * self.so], "little"),
                                 prefix + name + "/")
            elif 0x08 in types:
                self._datasets[prefix + name] = msgs

    def _btree_entries(self, addr, heap):
        a = self._abs(addr)
        if self.buf[a:a + 4] != b"TREE":
            raise H5FormatError("bad B-tree signature")
        ntype, level, used = self.buf[a + 4], self.buf[a + 5], self._u(a + 6, 2)
        if ntype != 0:
            raise H5FormatError("not a group B-tree")
        p = a + 8 + 2 * self.so  # after left/right sibling addresses
        out = []
        for i in range(used):
            child = self._u(p + self.sl, self.so)  # key i, child i
            p += self.sl + self.so
            if level > 0:
                out += self._btree_entries(child, heap)
            else:
                out += self._snod_entries(child, heap)
        return out

    def _snod_entries(self, addr, heap):
        a = self._abs(addr)
        if self.buf[a:a + 4] != b"SNOD":
            raise H5FormatError("bad symbol table node signature")
        n = self._u(a + 6, 2)
        out = []
        e = a + 8
        esize = 2 * self.so + 8 + 16
        for i in range(n):
            name_off = self._u(e, self.so)
            header = self._u(e + self.so, self.so)
            out.append((self._cstr(heap, name_off), header))
            e += esize
        return out

    # -- object headers
    def _object_messages(self, addr):
        a = self._abs(addr)
        if self.buf[a] != 1:
            raise H5FormatError("object header version %d not supported" % self.buf[a])
        nmsgs = self._u(a + 2, 2)
        size = self._u(a + 8, 4)
        blocks = [(a + 16, size)]
        msgs = []
        while blocks and len(msgs) < nmsgs:
            start, length = blocks.pop(0)
            p = start
            while p + 8 <= start + length and len(msgs) < nmsgs:
                mtype, msize = self._u(p, 2), self._u(p + 2, 2)
                data = self.buf[p + 8:p + 8 + msize]
                if mtype == 0x10:  # continuation
                    blocks.append((self._abs(int.from_bytes(data[:self.so], "little")),
                                   int.from_bytes(data[self.so:self.so + self.sl], "little")))
                msgs.append((mtype, data))
                p += 8 + msize
        return msgs

    # -- datasets
    def keys(self):
        return sorted(self._datasets)

    def __contains__(self, name):
        return name in self._datasets

    def __getitem__(self, name):
        msgs = dict(self._datasets[name])
        shape = self._dataspace(msgs[0x01])
        dtype = self._datatype(msgs[0x03])
        lay = msgs[0x08]
        ver = lay[0]
        n = int(np.prod(shape)) if shape else 1
        nbytes = n * dtype.itemsize
        if ver == 3:
            cls = lay[1]
            if cls == 1:  # contiguous: address, size
                addr = int.from_bytes(lay[2:2 + self.so], "little")
                size = int.from_bytes(lay[2 + self.so:2 + self.so + self.sl], "little")
                raw = self.buf[self._abs(addr):self._abs(addr) + size]
            elif cls == 0:  # compact: size, data
                size = int.from_bytes(lay[2:4], "little")
                raw = lay[4:4 + size]
            else:
                raise H5FormatError("chunked layout not supported")
        elif ver in (1, 2):
            rank, cls = lay[1], lay[2]
            if cls == 1:  # contiguous: address after 5 reserved bytes
                addr = int.from_bytes(lay[8:8 + self.so], "little")
                raw = self.buf[self._abs(addr):self._abs(addr) + nbytes]
            elif cls == 0:
                p = 8 + 4 * rank
                size = int.from_bytes(lay[p:p + 4], "little")
                raw = lay[p + 4:p + 4 + size]
            else:
                raise H5FormatError("chunked layout not supported")
        else:
            raise H5FormatError("layout message version %d not supported" % ver)
        arr = np.frombuffer(raw, dtype=dtype, count=n)
        return arr.reshape(shape) if shape else arr

    def _dataspace(self, d):
        ver, rank, flags = d[0], d[1], d[2]
        p = 8 if ver == 1 else 4
        return tuple(int.from_bytes(d[p + 8 * i:p + 8 * i + 8], "little") for i in range(rank))

    @staticmethod
    def _datatype(d):
        cls, ver = d[0] & 0x0F, d[0] >> 4
        bits = d[1] | (d[2] << 8) | (d[3] << 16)
        size = int.from_bytes(d[4:8], "little")
        order = ">" if bits & 1 else "<"
        if cls == 0:  # fixed point
            kind = "i" if bits & 0x8 else "u"
            return np.dtype(order + kind + str(size))
        if cls == 1:  # IEEE floating point
            if size not in (4, 8):
                raise H5FormatError("float of %d bytes" % size)
            return np.dtype(order + "f" + str(size))
        raise H5FormatError("datatype class %d not supported" % cls)
