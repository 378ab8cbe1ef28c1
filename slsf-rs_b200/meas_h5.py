"""Measurement files in carlo's `.meas.h5` layout, written without an HDF5 library.

write_theta_task_measurements (src/results.rs:55-105) writes, per task,

    /observables/<name>/bin_length   int64 scalar: the observable's internal bin length
    /observables/<name>/samples      float64 [n]: its bin means
    /version/carlo_version, /version/mc_package, /version/mc_version
                                     fixed-length ASCII strings (null-terminated padding)

through the hdf5-pure 0.21 crate; the dataframe tool of the reference reads
them back.  This module writes the same objects in the HDF5 file format
(HDF5 File Format Specification): a version 0 superblock, version 1 object
headers, groups as symbol tables (a version 1 B-tree of symbol table nodes
over a local heap of names, as many B-tree levels as a group needs), and datasets with a
version 1 dataspace, a version 1 datatype, a version 1 fill value message and
a version 2 contiguous layout.  The one difference from the reference's
files: `samples` is stored contiguously, without the chunking (1000) and
unlimited maximum shape the reference gives it, so a reader sees the same
values and shape but the dataset cannot be extended in place.

No HDF5 library is present in this image; the tests read these files back
with a reader written from the specification, which is itself checked
against a file libhdf5 wrote.
"""
import os
import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K = 4  # symbol table node: up to 2 * LEAF_K entries
INTERNAL_K = 16  # group B-tree node: up to 2 * INTERNAL_K children

# message types
_DATASPACE, _DATATYPE, _FILL, _LAYOUT, _SYMTAB, _NIL = 0x0001, 0x0003, 0x0005, 0x0008, 0x0011, 0x0000


class MeasH5Error(ValueError):
    pass


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _f64_type() -> bytes:
    # class 1 (floating point), version 1; little endian, implied mantissa MSB,
    # sign at bit 63; 8 bytes; offset 0, precision 64, exponent at 52 (11 bits),
    # mantissa at 0 (52 bits), bias 1023
    return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, 63, 0, 8, 0, 64, 52, 11, 0, 52, 1023)


def _i64_type() -> bytes:
    # class 0 (fixed point), version 1; little endian, signed; 8 bytes; offset 0, precision 64
    return struct.pack("<BBBBIHH", 0x10, 0x08, 0, 0, 8, 0, 64)


def _string_type(size: int) -> bytes:
    # class 3 (string), version 1; null-terminated padding, ASCII
    return struct.pack("<BBBBI", 0x13, 0x00, 0, 0, size)


def _dataspace(shape) -> bytes:
    return struct.pack("<BBBx4x", 1, len(shape), 0) + b"".join(struct.pack("<Q", d) for d in shape)


def _fill_value() -> bytes:
    # version 1: space allocated late, fill value written if set, defined, no value
    return struct.pack("<BBBBI", 1, 2, 2, 1, 0)


def _layout_contiguous(addr: int, shape, itemsize: int) -> bytes:
    # version 2, dimensionality = rank + 1 (the last dimension is the element size), class 1
    dims = tuple(shape) + (itemsize,)
    return struct.pack("<BBB5xQ", 2, len(dims), 1, addr) + b"".join(struct.pack("<I", d) for d in dims)


class _Writer:
    def __init__(self):
        self.buf = bytearray(96)  # the superblock is written last

    def alloc(self, data: bytes) -> int:
        addr = len(self.buf)
        self.buf += _pad8(bytes(data))
        return addr

    def object_header(self, messages) -> int:
        messages = list(messages)
        body = b"".join(messages)
        if len(body) < 32:  # libhdf5 allocates at least 32 bytes of messages
            messages.append(_message(_NIL, b"\0" * (32 - len(body) - 8)))
            body = b"".join(messages)
        # version 1, message count, reference count 1, message bytes; messages start 8-aligned
        return self.alloc(struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body)

    def dataset(self, dtype_msg: bytes, shape, raw: bytes, itemsize: int) -> int:
        data_addr = self.alloc(raw) if raw else UNDEF
        return self.object_header([
            _message(_FILL, _fill_value(), flags=1),
            _message(_DATATYPE, dtype_msg, flags=1),
            _message(_DATASPACE, _dataspace(shape)),
            _message(_LAYOUT, _layout_contiguous(data_addr, shape, itemsize), flags=1),
        ])

    def group(self, entries):
        """entries: [(name, object header address, (btree, heap) or None)];
        returns (object header, B-tree, heap) addresses of the new group."""
        if not entries:
            raise MeasH5Error("empty group")
        entries = sorted(entries, key=lambda e: e[0].encode("ascii"))
        names = [e[0] for e in entries]
        if len(set(names)) != len(names):
            raise MeasH5Error("duplicate names in one group")
        # local heap: "" at offset 0, then the names, then one free block
        data = bytearray(8)
        offsets = []
        for name in names:
            raw = name.encode("ascii")
            if not raw or b"\0" in raw or b"/" in raw:
                raise MeasH5Error(f"invalid object name {name!r}")
            offsets.append(len(data))
            data += _pad8(raw + b"\0")
        free_at = len(data)
        data += struct.pack("<QQ", 1, 16)  # last free block (next = 1), 16 bytes
        heap = len(self.buf)
        self.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(data), free_at, heap + 32))
        self.alloc(bytes(data))
        # symbol table nodes of up to 2K entries
        snods = []
        cap = 2 * LEAF_K
        for lo in range(0, len(entries), cap):
            part = list(zip(entries[lo:lo + cap], offsets[lo:lo + cap]))
            node = bytearray(b"SNOD" + struct.pack("<BxH", 1, len(part)))
            for (name, addr, stab), off in part:
                if stab is None:
                    node += struct.pack("<QQI4x16x", off, addr, 0)
                else:
                    node += struct.pack("<QQI4xQQ", off, addr, 1, *stab)
            node += b"\0" * (8 + 40 * cap - len(node))
            snods.append((self.alloc(bytes(node)), part[-1][1]))
        btree = self.btree(snods)
        header = self.object_header([_message(_SYMTAB, struct.pack("<QQ", btree, heap), flags=1)])
        return header, btree, heap

    def btree_node(self, level, children, left_key, left, right) -> int:
        """children: [(address, heap offset of the last name below it)]."""
        cap = 2 * INTERNAL_K
        node = bytearray(b"TREE" + struct.pack("<BBHQQ", 0, level, len(children), left, right))
        node += struct.pack("<Q", left_key)
        for addr, last in children:
            node += struct.pack("<QQ", addr, last)
        node += b"\0" * (24 + 8 * (2 * cap + 1) - len(node))
        return self.alloc(bytes(node))

    def btree(self, snods) -> int:
        """A group B-tree over its symbol table nodes, as many levels as the
        name count needs; the nodes of one level carry sibling addresses."""
        cap = 2 * INTERNAL_K
        node_size = 24 + 8 * (2 * cap + 1)
        children, level = snods, 0
        while len(children) > cap:
            parts = [children[lo:lo + cap] for lo in range(0, len(children), cap)]
            base = len(self.buf)  # this level's nodes are laid out back to back
            addrs = [base + k * node_size for k in range(len(parts))]
            nodes = []
            for k, part in enumerate(parts):
                left_key = 0 if k == 0 else parts[k - 1][-1][1]
                a = self.btree_node(level, part, left_key, addrs[k - 1] if k else UNDEF,
                                    addrs[k + 1] if k + 1 < len(parts) else UNDEF)
                assert a == addrs[k]
                nodes.append((a, part[-1][1]))
            children, level = nodes, level + 1
        return self.btree_node(level, children, 0, UNDEF, UNDEF)

    def finish(self, root) -> bytes:
        header, btree, heap = root
        sb = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, LEAF_K, INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, len(self.buf), UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, header, 1, btree, heap)
        assert len(sb) == 96
        self.buf[:96] = sb
        return bytes(self.buf)


def carlo_version() -> str:
    return os.environ.get("XY_CARLO_VERSION", "0.3.4")


def mc_version() -> str:
    return os.environ.get("XY_MC_VERSION", "0.1.0")


def encode_meas_h5(bins: dict) -> bytes:
    """bins: {observable name: (internal bin length, bin means)}, as
    write_theta_task_measurements takes them; the file's bytes."""
    if not bins:
        raise MeasH5Error("theta task result does not contain measurement bins")
    w = _Writer()
    observables = []
    for name, (bin_len, samples) in sorted(bins.items()):
        if int(bin_len) <= 0:
            raise MeasH5Error(f"{name}: internal bin length must be positive")
        s = np.ascontiguousarray(samples, dtype="<f8").ravel()
        if s.size == 0:
            raise MeasH5Error(f"{name}: no complete measurement bins to write")
        bl = w.dataset(_i64_type(), (), struct.pack("<q", int(bin_len)), 8)
        sm = w.dataset(_f64_type(), (s.size,), s.tobytes(), 8)
        g = w.group([("bin_length", bl, None), ("samples", sm, None)])
        observables.append((name, g[0], (g[1], g[2])))
    obs = w.group(observables)
    version = []
    for name, value in (("carlo_version", carlo_version()), ("mc_package", "SLSF.XYCarlo"),
                        ("mc_version", mc_version())):
        raw = value.encode("ascii")
        version.append((name, w.dataset(_string_type(len(raw)), (), raw, len(raw)), None))
    ver = w.group(version)
    root = w.group([("observables", obs[0], (obs[1], obs[2])), ("version", ver[0], (ver[1], ver[2]))])
    return w.finish(root)


def write_meas_h5(path, bins: dict) -> str:
    """write_theta_task_measurements_to_path (src/results.rs:55-105): the file
    goes to `<path>.tmp` first and is renamed into place."""
    data = encode_meas_h5(bins)
    path = os.fspath(path)
    parent = os.path.dirname(path)
    if parent:
        os.makedirs(parent, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(data)
    os.replace(tmp, path)
    return path


def write_job_measurements(records, bins_by_index: dict, output_dir) -> list:
    """write_theta_job_measurements (src/results.rs:38-53): one
    task<index + 1, 4 digits>/run0001.meas.h5 per task record."""
    paths = []
    for rec in records:
        k = rec.get("task_index", 0)
        bins = bins_by_index.get(k)
        if not bins:
            raise MeasH5Error("theta task result does not contain measurement bins")
        for name in bins:
            if name not in rec.get("observables", {}):
                raise MeasH5Error(f"missing observable estimate for {name}")
        path = os.path.join(os.fspath(output_dir), f"task{k + 1:04d}", "run0001.meas.h5")
        paths.append(write_meas_h5(path, bins))
    return paths
