"""A small HDF5 reader written from the published HDF5 File Format
Specification (version 0 superblock, version 1 object headers, symbol-table
groups, v1 B-trees, local heaps; dataspace, datatype, fill value, layout,
attribute and continuation messages), used by the tests to check files that
`slsf_rs_b200.meas_h5` writes.  No HDF5 library exists in this image, so the
reader is itself checked against a file libhdf5 wrote (a MATLAB 7.3 file that
ships with scipy's test data).

read(path) -> {"/path/to/dataset": Dataset, ...}; groups appear as Group
entries with their attributes.
"""
import struct
from dataclasses import dataclass, field

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5FormatError(ValueError):
    pass


@dataclass
class Dataset:
    shape: tuple
    maxshape: tuple
    dtype: object  # numpy dtype, or ("string", size, padding)
    layout: str
    chunks: tuple
    value: object
    attrs: dict = field(default_factory=dict)


@dataclass
class Group:
    attrs: dict = field(default_factory=dict)


class _File:
    def __init__(self, data: bytes):
        self.d = data
        self.base = None
        for off in [0] + [512 << k for k in range(12)]:
            if off + 8 <= len(data) and data[off:off + 8] == SIGNATURE:
                self.base = off
                break
        if self.base is None:
            raise H5FormatError("no HDF5 signature")
        p = self.base + 8
        ver = data[p]
        if ver not in (0, 1):
            raise H5FormatError(f"superblock version {ver} not supported")
        self.so, self.sl = data[p + 5], data[p + 6]
        if (self.so, self.sl) != (8, 8):
            raise H5FormatError("only 8-byte offsets and lengths are supported")
        self.leaf_k, self.internal_k = struct.unpack_from("<HH", data, p + 8)
        p += 16 if ver == 0 else 20
        base_addr, _free, self.eof, _drv = struct.unpack_from("<4Q", data, p)
        if base_addr != self.base:
            raise H5FormatError(f"base address {base_addr} != signature offset {self.base}")
        p += 32
        self.root = self.entry(p)

    # ---------------------------------------------------------------- helpers
    def at(self, addr):
        if addr == UNDEF:
            raise H5FormatError("undefined address")
        a = self.base + addr
        if a >= len(self.d):
            raise H5FormatError(f"address {addr} past the end of the file")
        return a

    def entry(self, p):
        name_off, header, cache = struct.unpack_from("<QQI", self.d, p)
        scratch = self.d[p + 24:p + 40]
        return {"name_off": name_off, "header": header, "cache": cache, "scratch": scratch}

    def heap_name(self, heap_addr, off):
        p = self.at(heap_addr)
        if self.d[p:p + 4] != b"HEAP":
            raise H5FormatError("bad local heap signature")
        size, _free, data_addr = struct.unpack_from("<QQQ", self.d, p + 8)
        if off >= size:
            raise H5FormatError("name offset outside the heap")
        q = self.at(data_addr) + off
        end = self.d.index(b"\0", q)
        return self.d[q:end].decode("ascii")

    # ---------------------------------------------------------------- groups
    def group_entries(self, btree_addr, heap_addr):
        """Symbol-table entries of a group in B-tree order."""
        out = []
        p = self.at(btree_addr)
        if self.d[p:p + 4] != b"TREE":
            raise H5FormatError("bad B-tree signature")
        ntype, level, used = self.d[p + 4], self.d[p + 5], struct.unpack_from("<H", self.d, p + 6)[0]
        if ntype != 0:
            raise H5FormatError("group B-tree of the wrong node type")
        if used > 2 * self.internal_k:
            raise H5FormatError("B-tree node over capacity")
        q = p + 24
        keys, children = [], []
        for i in range(used):
            keys.append(struct.unpack_from("<Q", self.d, q)[0])
            children.append(struct.unpack_from("<Q", self.d, q + 8)[0])
            q += 16
        keys.append(struct.unpack_from("<Q", self.d, q)[0])
        names_seen = []
        for i, child in enumerate(children):
            if level > 0:
                sub = self.group_entries(child, heap_addr)
            else:
                sub = self.snod(child, heap_addr)
            if sub:
                # key i+1 names the last entry of child i
                last = self.heap_name(heap_addr, keys[i + 1])
                if sub[-1][0] != last:
                    raise H5FormatError(f"B-tree key {last!r} != last entry {sub[-1][0]!r}")
            names_seen += [n for n, _ in sub]
            out += sub
        if names_seen != sorted(names_seen):
            raise H5FormatError("group entries are not in name order")
        return out

    def snod(self, addr, heap_addr):
        p = self.at(addr)
        if self.d[p:p + 4] != b"SNOD":
            raise H5FormatError("bad symbol table node signature")
        if self.d[p + 4] != 1:
            raise H5FormatError("symbol table node version")
        n = struct.unpack_from("<H", self.d, p + 6)[0]
        if n > 2 * self.leaf_k:
            raise H5FormatError("symbol table node over capacity")
        out = []
        for i in range(n):
            e = self.entry(p + 8 + 40 * i)
            out.append((self.heap_name(heap_addr, e["name_off"]), e))
        return out

    # ---------------------------------------------------------------- objects
    def messages(self, addr):
        p = self.at(addr)
        ver, _r, nmsg, _refc, size = struct.unpack_from("<BBHII", self.d, p)
        if ver != 1:
            raise H5FormatError(f"object header version {ver} not supported")
        blocks = [(p + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            q, size = blocks.pop(0)
            end = q + size
            while q + 8 <= end and len(out) < nmsg:
                mtype, msize, flags = struct.unpack_from("<HHB", self.d, q)
                body = self.d[q + 8:q + 8 + msize]
                if q + 8 + msize > end:
                    raise H5FormatError("message runs past its header block")
                if mtype == 0x10:
                    caddr, clen = struct.unpack_from("<QQ", body)
                    blocks.append((self.at(caddr), clen))
                out.append((mtype, flags, body))
                q += 8 + msize
        if len(out) != nmsg:
            raise H5FormatError(f"header holds {len(out)} of {nmsg} messages")
        return out

    def dataspace(self, b):
        ver, rank, flags = b[0], b[1], b[2]
        if ver == 1:
            p = 8
        elif ver == 2:
            p = 4
            if b[3] == 2:
                return None, None  # null dataspace
        else:
            raise H5FormatError(f"dataspace version {ver}")
        dims = struct.unpack_from(f"<{rank}Q", b, p)
        p += 8 * rank
        maxd = struct.unpack_from(f"<{rank}Q", b, p) if flags & 1 else dims
        return tuple(dims), tuple(None if m == UNDEF else m for m in maxd)

    def datatype(self, b):
        cls, ver = b[0] & 0x0F, b[0] >> 4
        bits = b[1] | (b[2] << 8) | (b[3] << 16)
        size = struct.unpack_from("<I", b, 4)[0]
        if ver not in (1, 2, 3):
            raise H5FormatError(f"datatype version {ver}")
        if cls == 0:  # fixed-point
            order = ">" if bits & 1 else "<"
            signed = bool(bits & 8)
            offset, precision = struct.unpack_from("<HH", b, 8)
            if offset != 0 or precision != 8 * size:
                raise H5FormatError("padded integers are not supported")
            return np.dtype(f"{order}{'i' if signed else 'u'}{size}")
        if cls == 1:  # floating-point
            order = ">" if bits & 1 else "<"
            offset, precision, eloc, esize, mloc, msize, bias = struct.unpack_from("<HHBBBBI", b, 8)
            ieee = {4: (0, 32, 23, 8, 0, 23, 127, 31), 8: (0, 64, 52, 11, 0, 52, 1023, 63)}
            if size not in ieee or (offset, precision, eloc, esize, mloc, msize, bias, (bits >> 8) & 0xFF) != \
                    ieee[size] or ((bits >> 4) & 3) != 2:
                raise H5FormatError("non-IEEE floating-point type")
            return np.dtype(f"{order}f{size}")
        if cls == 3:  # string
            return ("string", size, bits & 0x0F, (bits >> 4) & 0x0F)
        raise H5FormatError(f"datatype class {cls} not supported")

    def read_object(self, addr):
        shape = maxshape = dtype = layout = None
        chunks, value, attrs, symtab = (), None, {}, None
        raw = None
        for mtype, _flags, b in self.messages(addr):
            if mtype == 0x0001:
                shape, maxshape = self.dataspace(b)
            elif mtype == 0x0003:
                dtype = self.datatype(b)
            elif mtype == 0x0008:
                raw = b
            elif mtype == 0x0011:
                symtab = struct.unpack_from("<QQ", b)
            elif mtype == 0x000C:
                name, val = self.attribute(b)
                attrs[name] = val
        if symtab is not None:
            return Group(attrs), symtab
        if raw is None or dtype is None or shape is None:
            raise H5FormatError("object is neither a group nor a dataset")
        layout, chunks, value = self.layout(raw, shape, dtype)
        return Dataset(shape, maxshape, dtype, layout, chunks, value, attrs), None

    def attribute(self, b):
        ver = b[0]
        if ver != 1:
            raise H5FormatError(f"attribute version {ver}")
        nsize, tsize, ssize = struct.unpack_from("<HHH", b, 2)
        p = 8
        name = b[p:p + nsize].split(b"\0")[0].decode("ascii")
        p += (nsize + 7) // 8 * 8
        dtype = self.datatype(b[p:p + tsize])
        p += (tsize + 7) // 8 * 8
        shape, _ = self.dataspace(b[p:p + ssize])
        p += (ssize + 7) // 8 * 8
        return name, self.decode(b[p:], shape, dtype)

    def decode(self, raw, shape, dtype):
        n = int(np.prod(shape)) if shape else 1
        if isinstance(dtype, tuple):
            size = dtype[1]
            vals = [raw[i * size:(i + 1) * size] for i in range(n)]
            vals = [v.split(b"\0")[0].rstrip(b" ").decode("ascii") if dtype[2] in (0, 1, 2) else v for v in vals]
            return vals[0] if not shape else np.array(vals, dtype=object).reshape(shape)
        a = np.frombuffer(raw[:n * dtype.itemsize], dtype=dtype)
        if a.size != n:
            raise H5FormatError("data shorter than its dataspace")
        return a[0] if not shape else a.reshape(shape)

    def layout(self, b, shape, dtype):
        itemsize = dtype[1] if isinstance(dtype, tuple) else dtype.itemsize
        n = int(np.prod(shape)) if shape else 1
        if b[0] in (1, 2):
            # version 1/2: dimensionality, class, 5 reserved, [address], dims (the
            # last one the element size), [compact size + data]
            nd, cls = b[1], b[2]
            p = 8
            addr = None
            if cls != 0:
                addr = struct.unpack_from("<Q", b, p)[0]
                p += 8
            dims = struct.unpack_from(f"<{nd}I", b, p)
            p += 4 * nd
            if cls == 0:
                size = struct.unpack_from("<I", b, p)[0]
                return "compact", (), self.decode(b[p + 4:p + 4 + size], shape, dtype)
            if cls == 1:
                size = int(np.prod(dims))
                if size != n * itemsize:
                    raise H5FormatError("contiguous storage size does not match the dataspace")
                q = self.at(addr)
                return "contiguous", (), self.decode(self.d[q:q + size], shape, dtype)
            raise H5FormatError("chunked layout of version 1/2 is not supported")
        if b[0] != 3:
            raise H5FormatError(f"layout version {b[0]} not supported")
        cls = b[1]
        if cls == 0:  # compact
            size = struct.unpack_from("<H", b, 2)[0]
            return "compact", (), self.decode(b[4:4 + size], shape, dtype)
        if cls == 1:  # contiguous
            addr, size = struct.unpack_from("<QQ", b, 2)
            if size != n * itemsize:
                raise H5FormatError("contiguous storage size does not match the dataspace")
            if addr == UNDEF:
                raise H5FormatError("contiguous storage never allocated")
            p = self.at(addr)
            return "contiguous", (), self.decode(self.d[p:p + size], shape, dtype)
        if cls == 2:  # chunked, v1 B-tree of type 1
            nd = b[2]
            btree = struct.unpack_from("<Q", b, 3)[0]
            dims = struct.unpack_from(f"<{nd}I", b, 11)
            chunk, elem = dims[:-1], dims[-1]
            if elem != itemsize or len(chunk) != len(shape):
                raise H5FormatError("chunk dimensions do not match the dataset")
            out = np.zeros(n * itemsize, dtype=np.uint8).reshape(*shape, itemsize) if shape else None
            for offs, caddr, csize in self.chunk_index(btree, nd):
                if csize != int(np.prod(chunk)) * itemsize:
                    raise H5FormatError("filtered chunks are not supported")
                p = self.at(caddr)
                blk = np.frombuffer(self.d[p:p + csize], dtype=np.uint8).reshape(*chunk, itemsize)
                sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunk, shape))
                out[sl] = blk[tuple(slice(0, s.stop - s.start) for s in sl)]
            return "chunked", tuple(chunk), self.decode(out.tobytes(), shape, dtype)
        raise H5FormatError(f"layout class {cls}")

    def chunk_index(self, addr, nd):
        p = self.at(addr)
        if self.d[p:p + 4] != b"TREE" or self.d[p + 4] != 1:
            raise H5FormatError("bad chunk B-tree node")
        level, used = self.d[p + 5], struct.unpack_from("<H", self.d, p + 6)[0]
        ksize = 8 + 8 * nd
        q = p + 24
        out = []
        for i in range(used):
            csize, _mask = struct.unpack_from("<II", self.d, q)
            offs = struct.unpack_from(f"<{nd}Q", self.d, q + 8)
            child = struct.unpack_from("<Q", self.d, q + ksize)[0]
            if level > 0:
                out += self.chunk_index(child, nd)
            else:
                out.append((offs[:-1], child, csize))
            q += ksize + 8
        return out


def read(path):
    with open(path, "rb") as f:
        h = _File(f.read())
    out = {}

    def walk(prefix, obj_addr):
        obj, symtab = h.read_object(obj_addr)
        out[prefix or "/"] = obj
        if symtab is None:
            return
        btree, heap = symtab
        for name, e in h.group_entries(btree, heap):
            walk(f"{prefix}/{name}", e["header"])

    walk("", h.root["header"])
    return out
