"""A small read-only HDF5 reader for the files of the contact-scene-v1 package (the FCLIB
local-problem copies, data/ncp/scenes/NN.hdf5), written from the published HDF5 file-format
specification because h5py is not installed in this image.

What it reads: superblock version 0 or 1 (8-byte offsets and lengths), version-1 object
headers with continuation blocks, old-style groups (symbol-table message, version-1 B-tree of
group nodes, symbol-table nodes, local heap), and datasets of little- or big-endian integers and
IEEE floats with a simple dataspace, stored compact, contiguous or chunked (version-1 B-tree
chunk index) with the deflate and shuffle filters; attributes (version 1) of those types (other
attribute types are listed with the value None).  Other layouts raise NotImplementedError.

    f = H5File(path)
    f["fclib_local/W/x"]            # numpy array
    f.attrs("fclib_local/W")        # {name: value}
"""
from __future__ import annotations

import zlib

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5File:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.buf = f.read()
        b = self.buf
        if b[:8] != _SIG:
            raise ValueError(f"{path}: not an HDF5 file")
        ver = b[8]
        if ver not in (0, 1):
            raise NotImplementedError(f"{path}: superblock version {ver}")
        self.so, self.sl = b[13], b[14]
        if (self.so, self.sl) != (8, 8):
            raise NotImplementedError("only 8-byte offsets and lengths")
        pos = 24 if ver == 0 else 28  # after the fixed fields (v1 adds the indexed-storage K)
        pos += 4 * 8  # base, free-space, end-of-file, driver-info addresses
        self.root = self._u(pos + 8, 8)  # root symbol-table entry: link name offset, object header
        self._cache = {}

    # ---- primitives ----
    def _u(self, pos, n):
        return int.from_bytes(self.buf[pos:pos + n], "little")

    def _messages(self, addr):
        """(type, flags, data bytes) of every message of a version-1 object header."""
        b = self.buf
        if b[addr] != 1:
            raise NotImplementedError(f"object header version {b[addr]} at {addr:#x}")
        n_msgs = self._u(addr + 2, 2)
        size = self._u(addr + 8, 4)
        blocks = [(addr + 16, size)]  # header prefix 12 bytes + 4 of alignment
        out = []
        while blocks and len(out) < n_msgs:
            start, length = blocks.pop(0)
            pos, end = start, start + length
            while pos + 8 <= end and len(out) < n_msgs:
                mtype, msize, mflags = self._u(pos, 2), self._u(pos + 2, 2), b[pos + 4]
                data = b[pos + 8:pos + 8 + msize]
                out.append((mtype, mflags, data))
                if mtype == 0x10:  # continuation: more messages elsewhere
                    blocks.append((int.from_bytes(data[0:8], "little"), int.from_bytes(data[8:16], "little")))
                pos += 8 + msize
        return out

    # ---- groups ----
    def _heap_name(self, heap, off):
        b = self.buf
        if b[heap:heap + 4] != b"HEAP":
            raise ValueError("bad local heap")
        data = self._u(heap + 24, 8)
        end = b.index(b"\0", data + off)
        return b[data + off:end].decode()

    def _group_entries(self, addr):
        """{name: object header address} of an old-style group."""
        st = [d for t, _, d in self._messages(addr) if t == 0x11]
        if not st:
            raise NotImplementedError(f"object at {addr:#x} is not an old-style group")
        btree, heap = int.from_bytes(st[0][0:8], "little"), int.from_bytes(st[0][8:16], "little")
        out = {}
        self._walk_group_tree(btree, heap, out)
        return out

    def _walk_group_tree(self, node, heap, out):
        b = self.buf
        if b[node:node + 4] != b"TREE" or b[node + 4] != 0:
            raise ValueError("bad group B-tree node")
        level, used = b[node + 5], self._u(node + 6, 2)
        pos = node + 24 + 8  # signature, type, level, used, siblings; then key 0
        for _ in range(used):
            child = self._u(pos, 8)
            pos += 16  # child address, next key
            if level > 0:
                self._walk_group_tree(child, heap, out)
                continue
            if b[child:child + 4] != b"SNOD":
                raise ValueError("bad symbol-table node")
            n = self._u(child + 6, 2)
            e = child + 8
            for _ in range(n):
                out[self._heap_name(heap, self._u(e, 8))] = self._u(e + 8, 8)
                e += 40

    def _lookup(self, path):
        addr = self.root
        for part in [p for p in path.strip("/").split("/") if p]:
            addr = self._group_entries(addr)[part]
        return addr

    def keys(self, path="/"):
        return sorted(self._group_entries(self._lookup(path)))

    # ---- datatypes, dataspaces, data ----
    @staticmethod
    def _dtype(d):
        cls, size = d[0] & 0x0F, int.from_bytes(d[4:8], "little")
        big = d[1] & 1
        end = ">" if big else "<"
        if cls == 0:
            signed = (d[1] >> 3) & 1
            return np.dtype(f"{end}{'i' if signed else 'u'}{size}")
        if cls == 1:
            return np.dtype(f"{end}f{size}")
        raise NotImplementedError(f"datatype class {cls}")

    @staticmethod
    def _shape(d):
        ver, rank, flags = d[0], d[1], d[2]
        pos = 8 if ver == 1 else 4
        if ver == 2 and d[3] == 0:  # scalar
            return ()
        dims = [int.from_bytes(d[pos + 8 * i:pos + 8 * i + 8], "little") for i in range(rank)]
        return tuple(dims)

    def _chunks(self, node, rank, out, csize, dtype, shape, filters):
        b = self.buf
        if b[node:node + 4] != b"TREE" or b[node + 4] != 1:
            raise ValueError("bad chunk B-tree node")
        level, used = b[node + 5], self._u(node + 6, 2)
        ksize = 8 + 8 * (rank + 1)
        pos = node + 24
        for _ in range(used):
            nbytes, mask = self._u(pos, 4), self._u(pos + 4, 4)
            offs = [self._u(pos + 8 + 8 * i, 8) for i in range(rank)]
            child = self._u(pos + ksize, 8)
            if level > 0:
                self._chunks(child, rank, out, csize, dtype, shape, filters)
            else:
                raw = b[child:child + nbytes]
                for fid in reversed(filters):
                    if mask & (1 << filters.index(fid)):
                        continue
                    if fid == 1:
                        raw = zlib.decompress(raw)
                    elif fid == 2:
                        n = len(raw) // dtype.itemsize
                        raw = np.frombuffer(raw, np.uint8).reshape(dtype.itemsize, n).T.tobytes()
                    else:
                        raise NotImplementedError(f"filter {fid}")
                blk = np.frombuffer(raw, dtype)[:int(np.prod(csize))].reshape(csize)
                sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, csize, shape))
                out[sl] = blk[tuple(slice(0, x.stop - x.start) for x in sl)]
            pos += ksize + 8

    def __getitem__(self, path):
        if path in self._cache:
            return self._cache[path]
        msgs = self._messages(self._lookup(path))
        by = {}
        for t, _, d in msgs:
            by.setdefault(t, d)
        shape, dtype, lay = self._shape(by[0x01]), self._dtype(by[0x03]), by[0x08]
        filters = []
        if 0x0B in by:
            f = by[0x0B]
            nf, pos = f[1], 8 if f[0] == 1 else 2
            for _ in range(nf):
                fid = int.from_bytes(f[pos:pos + 2], "little")
                if f[0] == 1 or fid >= 256:
                    nlen = int.from_bytes(f[pos + 2:pos + 4], "little")
                    ncl = int.from_bytes(f[pos + 6:pos + 8], "little")
                    pos += 8 + ((nlen + 7) // 8 * 8 if f[0] == 1 else nlen) + 4 * ncl
                    if f[0] == 1 and ncl % 2:
                        pos += 4
                else:
                    ncl = int.from_bytes(f[pos + 4:pos + 6], "little")
                    pos += 6 + 4 * ncl
                filters.append(fid)
        if lay[0] != 3:
            raise NotImplementedError(f"data layout version {lay[0]}")
        n = int(np.prod(shape)) if shape else 1
        if lay[1] == 0:  # compact
            size = int.from_bytes(lay[2:4], "little")
            arr = np.frombuffer(lay[4:4 + size], dtype)[:n].reshape(shape)
        elif lay[1] == 1:  # contiguous
            addr = int.from_bytes(lay[2:10], "little")
            arr = (np.zeros(shape, dtype) if addr == UNDEF else
                   np.frombuffer(self.buf, dtype, count=n, offset=addr).reshape(shape))
        elif lay[1] == 2:  # chunked, version-1 B-tree index
            rank = lay[2]
            btree = int.from_bytes(lay[3:11], "little")
            csize = tuple(int.from_bytes(lay[11 + 4 * i:15 + 4 * i], "little") for i in range(rank - 1))
            arr = np.zeros(shape, dtype)
            if btree != UNDEF:
                self._chunks(btree, rank - 1, arr, csize, dtype, shape, filters)
        else:
            raise NotImplementedError(f"layout class {lay[1]}")
        out = np.array(arr, dtype=dtype.newbyteorder("="))
        self._cache[path] = out
        return out

    def attrs(self, path):
        """Attributes (version-1 messages) of the object at `path`."""
        out = {}
        for t, _, d in self._messages(self._lookup(path)):
            if t != 0x0C:
                continue
            if d[0] != 1:
                raise NotImplementedError(f"attribute message version {d[0]}")
            nl, tl, sl = (int.from_bytes(d[2 + 2 * i:4 + 2 * i], "little") for i in range(3))
            pad = lambda x: (x + 7) // 8 * 8
            pos = 8
            name = d[pos:pos + nl].rstrip(b"\0").decode()
            pos += pad(nl)
            try:
                dt = self._dtype(d[pos:pos + tl])
            except NotImplementedError:  # strings and other classes: named, value not read
                out[name] = None
                continue
            pos += pad(tl)
            shp = self._shape(d[pos:pos + sl])
            pos += pad(sl)
            n = int(np.prod(shp)) if shp else 1
            val = np.frombuffer(d[pos:pos + n * dt.itemsize], dt).reshape(shp)
            out[name] = val.item() if val.size == 1 else val.copy()
        return out
