"""A minimal read-only HDF5 reader, written from the public HDF5 file-format
specification, for the files this project needs to read without h5py (not
installed here): superblock version 0, groups stored as symbol tables (v1
B-trees of SNOD nodes with a local heap), version-1 object headers, datasets
of little-endian IEEE floats / integers with a contiguous, compact or chunked
(deflate / shuffle) layout.

    data = read_h5(path)       # {"rho/SNAPSHOT1": ndarray, "time/sim_time": ndarray, ...}

Test infrastructure only (it generates fixtures); nothing in the product
imports it.
"""
from __future__ import annotations

import zlib

import numpy as np


class _File:
    def __init__(self, buf: bytes):
        self.b = buf
        if buf[:8] != b"\x89HDF\r\n\x1a\n":
            raise ValueError("not an HDF5 file")
        if buf[8] != 0:
            raise ValueError(f"superblock version {buf[8]} not supported")
        self.so = buf[13]            # size of offsets
        self.sl = buf[14]            # size of lengths
        if self.so != 8 or self.sl != 8:
            raise ValueError("only 8-byte offsets and lengths are supported")
        # 24 fixed bytes, then base, free-space, end-of-file and driver addresses
        self.base = self.u(24, 8)
        self.root = 24 + 4 * 8       # root group symbol-table entry

    def u(self, off, n):
        return int.from_bytes(self.b[off:off + n], "little")

    # ---- symbol-table entries, object headers --------------------------------
    def entry(self, off):
        """(link-name offset, object-header address, cache type, scratch pad)."""
        return self.u(off, 8), self.u(off + 8, 8), self.u(off + 16, 4), self.b[off + 24:off + 40]

    def messages(self, addr):
        """The (type, data) messages of a version-1 object header."""
        b = self.b
        if b[addr] != 1:
            raise ValueError(f"object header version {b[addr]} not supported")
        nmsg = self.u(addr + 2, 2)
        size = self.u(addr + 8, 4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p, end = start, start + length
            while p + 8 <= end and len(out) < nmsg:
                mtype, msize = self.u(p, 2), self.u(p + 2, 2)
                data = b[p + 8:p + 8 + msize]
                if mtype == 0x0010:   # continuation: (offset, length) of more messages
                    blocks.append((int.from_bytes(data[:8], "little"), int.from_bytes(data[8:16], "little")))
                out.append((mtype, data))
                p += 8 + msize
        return out

    # ---- groups ----------------------------------------------------------------
    def heap_name(self, heap, off):
        if self.b[heap:heap + 4] != b"HEAP":
            raise ValueError("bad local heap")
        data = self.u(heap + 24, 8)
        s = data + off
        return self.b[s:self.b.index(b"\0", s)].decode()

    def group_children(self, btree, heap):
        """name -> object-header address for a symbol-table group."""
        out = {}
        stack = [btree]
        while stack:
            node = stack.pop()
            sig = self.b[node:node + 4]
            if sig == b"TREE":         # internal or leaf node: its children are nodes or SNODs
                used = self.u(node + 6, 2)
                p = node + 8 + 16          # after left / right sibling addresses
                p += 8                     # key 0
                for _ in range(used):
                    child = self.u(p, 8)
                    p += 16                # child address, next key
                    stack.append(child)
            elif sig == b"SNOD":
                n = self.u(node + 6, 2)
                for k in range(n):
                    name_off, obj, _, _ = self.entry(node + 8 + 40 * k)
                    out[self.heap_name(heap, name_off)] = obj
            else:
                raise ValueError("bad group node")
        return out

    # ---- datasets ----------------------------------------------------------------
    def dataset(self, msgs):
        shape = dtype = layout = None
        filters = []
        for mtype, d in msgs:
            if mtype == 0x0001:                     # dataspace
                ver, rank = d[0], d[1]
                off = 8 if ver == 1 else 4
                shape = tuple(int.from_bytes(d[off + 8 * i:off + 8 * i + 8], "little") for i in range(rank))
            elif mtype == 0x0003:                   # datatype
                cls = d[0] & 0x0F
                size = int.from_bytes(d[4:8], "little")
                big = bool(d[1] & 1)
                if cls == 1:
                    dtype = np.dtype(("<" if not big else ">") + "f" + str(size))
                elif cls == 0:
                    signed = bool(d[1] & 0x08)
                    dtype = np.dtype(("<" if not big else ">") + ("i" if signed else "u") + str(size))
                else:
                    raise ValueError(f"datatype class {cls} not supported")
            elif mtype == 0x0008:                   # data layout
                layout = d
            elif mtype == 0x000B:                   # filter pipeline
                filters = self.filter_ids(d)
        if shape is None or dtype is None or layout is None:
            return None
        n = int(np.prod(shape)) if shape else 1
        ver = layout[0]
        if ver == 3:
            cls = layout[1]
            if cls == 0:                            # compact
                size = int.from_bytes(layout[2:4], "little")
                raw = layout[4:4 + size]
            elif cls == 1:                          # contiguous
                addr = int.from_bytes(layout[2:10], "little")
                raw = self.b[addr:addr + n * dtype.itemsize]
            elif cls == 2:                          # chunked
                rank = layout[2]
                addr = int.from_bytes(layout[3:11], "little")
                cdims = [int.from_bytes(layout[11 + 4 * i:15 + 4 * i], "little") for i in range(rank)]
                return self.chunked(addr, shape, cdims[:-1], dtype, filters)
            else:
                raise ValueError("layout class not supported")
        else:
            raise ValueError(f"layout version {ver} not supported")
        return np.frombuffer(raw, dtype=dtype, count=n).reshape(shape).astype(dtype.newbyteorder("="))

    @staticmethod
    def filter_ids(d):
        ver, nf = d[0], d[1]
        p = 8 if ver == 1 else 2
        ids = []
        for _ in range(nf):
            fid = int.from_bytes(d[p:p + 2], "little")
            if ver == 1 or fid >= 256:
                name_len = int.from_bytes(d[p + 2:p + 4], "little")
                nvals = int.from_bytes(d[p + 6:p + 8], "little")
                p += 8 + ((name_len + 7) // 8) * 8 + 4 * nvals + (4 if (ver == 1 and nvals % 2) else 0)
            else:
                nvals = int.from_bytes(d[p + 4:p + 6], "little")
                p += 6 + 4 * nvals
            ids.append(fid)
        return ids

    def chunked(self, btree, shape, cdims, dtype, filters):
        out = np.zeros(shape, dtype=dtype)
        rank = len(shape)
        stack = [btree]
        while stack:
            node = stack.pop()
            if self.b[node:node + 4] != b"TREE":
                raise ValueError("bad chunk index node")
            level = self.b[node + 5]
            used = self.u(node + 6, 2)
            p = node + 24
            keysize = 8 + 8 * (rank + 1)
            for _ in range(used):
                csize = self.u(p, 4)
                offs = [self.u(p + 8 + 8 * i, 8) for i in range(rank)]
                child = self.u(p + keysize, 8)
                p += keysize + 8
                if level > 0:
                    stack.append(child)
                    continue
                raw = self.b[child:child + csize]
                for fid in reversed(filters):
                    if fid == 1:
                        raw = zlib.decompress(raw)
                    elif fid == 2:
                        a = np.frombuffer(raw, dtype=np.uint8).reshape(dtype.itemsize, -1)
                        raw = a.T.tobytes()
                    else:
                        raise ValueError(f"filter {fid} not supported")
                chunk = np.frombuffer(raw, dtype=dtype).reshape(cdims)
                sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
                out[sl] = chunk[tuple(slice(0, x.stop - x.start) for x in sl)]
        return out


def read_h5(path: str) -> dict:
    """Every dataset of the file, keyed by its path ("group/name")."""
    with open(path, "rb") as fh:
        f = _File(fh.read())
    out = {}
    _, root_obj, _, _ = f.entry(f.root)
    stack = [("", root_obj)]
    while stack:
        prefix, obj = stack.pop()
        msgs = f.messages(obj)
        stab = [d for t, d in msgs if t == 0x0011]
        if stab:
            btree = int.from_bytes(stab[0][:8], "little")
            heap = int.from_bytes(stab[0][8:16], "little")
            for name, child in f.group_children(btree, heap).items():
                stack.append((prefix + name + "/", child))
        else:
            arr = f.dataset(msgs)
            if arr is not None:
                out[prefix.rstrip("/")] = arr
    return out
