"""HDF5 halo catalogues without libhdf5.

write_catalog_hdf5 mirrors PeakPatch.write_catalog_hdf5 (ext/HDF5Ext.jl:47-104)
through libppb.so; read_catalog_hdf5 reads back the subset of the HDF5 file
format that writer produces and other simple files share: superblock
version 0 or 1, groups held by a version 1 B-tree with symbol table nodes and
a local heap of names, version 1 object headers, simple dataspaces (version 1
or 2) of IEEE floats or integers with contiguous storage.  Anything outside
that subset raises ValueError."""
from __future__ import annotations

import ctypes
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


def write_catalog_hdf5(path: str, records: np.ndarray, Om: float, OL: float, h: float, z_max: float = 10.0) -> None:
    """The catalogue's columns (x, y, z, ra, dec, redshift, chi, M200m, RTHL,
    vx, vy, vz, and for 33-field records vx2, vy2, vz2, overdensity, e_v,
    p_v, Rf, zform) as Float32 datasets.  Om is the total matter density."""
    from . import _p, load_library
    rec = np.ascontiguousarray(records, dtype=np.float32)
    n, nf = (rec.shape[0], rec.shape[1]) if rec.ndim == 2 else (0, 11)
    rc = load_library().ppb_write_catalog_hdf5(path.encode(), _p(rec) if n else None, n, nf, Om, OL, h, z_max)
    if rc != 0:
        raise OSError(f"ppb_write_catalog_hdf5 failed ({rc}) for {path}")


class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        if data[:8] != b"\x89HDF\r\n\x1a\n":
            raise ValueError("not an HDF5 file (signature)")
        ver = data[8]
        if ver not in (0, 1):
            raise ValueError(f"superblock version {ver} is outside the supported subset")
        if data[13] != 8 or data[14] != 8:
            raise ValueError("only 8-byte offsets and lengths are supported")
        self.leaf_k, self.int_k = struct.unpack_from("<HH", data, 16)
        p = 24 + (4 if ver == 1 else 0)
        base, _, eof, _ = struct.unpack_from("<QQQQ", data, p)
        if base != 0:
            raise ValueError("non-zero base address")
        if eof > len(data):
            raise ValueError("file shorter than its end-of-file address")
        self.root = p + 32   # root group symbol table entry

    def u64(self, at):
        return struct.unpack_from("<Q", self.d, at)[0]

    def entry(self, at):
        name_off, obj, cache = struct.unpack_from("<QQI", self.d, at)
        scratch = struct.unpack_from("<QQ", self.d, at + 24)
        return name_off, obj, cache, scratch

    def messages(self, at):
        ver, _, nmsg, _, size = struct.unpack_from("<BBHII", self.d, at)
        if ver != 1:
            raise ValueError(f"object header version {ver} is outside the supported subset")
        out, p, end = [], at + 16, at + 16 + size
        while p < end and len(out) < nmsg:
            mtype, msize, flags = struct.unpack_from("<HHB", self.d, p)
            out.append((mtype, p + 8, msize))
            p += 8 + msize
            if mtype == 0x0010:   # continuation: further messages elsewhere
                raise ValueError("object header continuation is outside the supported subset")
        return out

    def heap_name(self, heap, off):
        if self.d[heap:heap + 4] != b"HEAP":
            raise ValueError("bad local heap")
        seg = self.u64(heap + 24)
        end = self.d.index(b"\0", seg + off)
        return self.d[seg + off:end].decode()

    def group(self, btree, heap):
        out = {}
        if self.d[btree:btree + 4] != b"TREE" or self.d[btree + 4] != 0:
            raise ValueError("bad group B-tree node")
        level, used = self.d[btree + 5], struct.unpack_from("<H", self.d, btree + 6)[0]
        for i in range(used):
            child = self.u64(btree + 24 + 8 + 16 * i)
            if level > 0:
                out.update(self.group(child, heap))
                continue
            if self.d[child:child + 4] != b"SNOD":
                raise ValueError("bad symbol table node")
            nsym = struct.unpack_from("<H", self.d, child + 6)[0]
            for s in range(nsym):
                name_off, obj, _, _ = self.entry(child + 8 + 40 * s)
                out[self.heap_name(heap, name_off)] = obj
        return out

    def dataset(self, obj):
        shape = dtype = addr = size = None
        for mtype, p, _ in self.messages(obj):
            if mtype == 0x0001:
                ver, rank, flags = self.d[p], self.d[p + 1], self.d[p + 2]
                q = p + (8 if ver == 1 else 4)
                shape = tuple(self.u64(q + 8 * r) for r in range(rank))
            elif mtype == 0x0003:
                cls, b0 = self.d[p] & 0x0F, self.d[p + 1]
                sz = struct.unpack_from("<I", self.d, p + 4)[0]
                if b0 & 1:
                    raise ValueError("big-endian data is outside the supported subset")
                if cls == 1:
                    dtype = {4: "<f4", 8: "<f8"}[sz]
                elif cls == 0:
                    dtype = ("<i" if b0 & 8 else "<u") + str(sz)
                else:
                    raise ValueError(f"datatype class {cls} is outside the supported subset")
            elif mtype == 0x0008:
                if self.d[p] != 3 or self.d[p + 1] != 1:
                    raise ValueError("only contiguous layout (message version 3) is supported")
                addr, size = self.u64(p + 2), self.u64(p + 10)
        if shape is None or dtype is None or size is None:
            raise ValueError("dataset without dataspace, datatype or layout")
        count = int(np.prod(shape)) if shape else 1
        if count == 0 or addr == UNDEF:
            return np.zeros(shape, dtype)
        if size != count * np.dtype(dtype).itemsize:
            raise ValueError("storage size does not match the dataspace")
        return np.frombuffer(self.d, dtype=dtype, count=count, offset=addr).reshape(shape).copy()

    def root_datasets(self):
        _, obj, cache, scratch = self.entry(self.root)
        btree = heap = None
        for mtype, p, _ in self.messages(obj):
            if mtype == 0x0011:
                btree, heap = self.u64(p), self.u64(p + 8)
        if btree is None:
            if cache == 1:
                btree, heap = scratch
            else:
                raise ValueError("root group without a symbol table")
        return {name: self.dataset(o) for name, o in self.group(btree, heap).items()}


def read_catalog_hdf5(path: str) -> dict:
    """The root group's datasets as numpy arrays, by name."""
    with open(path, "rb") as f:
        return _Reader(f.read()).root_datasets()
