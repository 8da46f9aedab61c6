"""Minimal HDF5 writer for Nebula ``.mat`` material files.

Nebula reads its per-material scattering tables from HDF5 files
(``source/io/hdf5_file.cpp``: root attributes that are either a
variable-length string or a compound ``{double value; vlen string unit}``,
float/double datasets with a ``units`` attribute, and axes attached as HDF5
dimension scales).  libhdf5/h5py are not available in this environment, so
this module writes exactly that subset of the HDF5 file format, following the
public HDF5 File Format Specification (version 0 superblock, version 1 object
headers, symbol-table groups with a v1 B-tree and a local heap, contiguous
dataset storage, one global heap collection for variable-length data).  These
are the structures libhdf5 emits for files created with the default
("earliest") format bounds, which is how h5py/cstool write ``.mat`` files.

The matching reader is ``nebula_b200/csrc/h5lite.cpp``.
"""
from __future__ import annotations

import struct
from collections import OrderedDict

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
LEAF_K = 32          # symbol-table-node capacity is 2*LEAF_K entries
INTERNAL_K = 16      # v1 B-tree node capacity is 2*INTERNAL_K children
HEAP_FREE_NULL = 1   # "no next free block" marker in a local-heap free list
GCOL_MIN = 4096


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * ((-len(b)) % 8)


# --------------------------------------------------------------------------
# Datatype messages (HDF5 spec IV.A.2.d)
# --------------------------------------------------------------------------
def dt_float(size: int) -> bytes:
    if size == 4:
        return struct.pack("<B3BI", 0x11, 0x20, 31, 0, 4) + struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
    return struct.pack("<B3BI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)


def dt_int(size: int, signed: bool) -> bytes:
    return struct.pack("<B3BI", 0x10, 0x08 if signed else 0x00, 0, 0, size) + struct.pack("<HH", 0, 8 * size)


def dt_fixed_string(n: int) -> bytes:
    return struct.pack("<B3BI", 0x13, 0x00, 0, 0, n)


def dt_vlen_string() -> bytes:
    # variable-length, type=string (1), padding=null-terminate, charset=ascii
    return struct.pack("<B3BI", 0x19, 0x01, 0x00, 0, 16) + dt_int(1, False)


def dt_objref() -> bytes:
    return struct.pack("<B3BI", 0x17, 0x00, 0, 0, 8)


def dt_vlen_sequence(base: bytes) -> bytes:
    return struct.pack("<B3BI", 0x19, 0x00, 0x00, 0, 16) + base


def dt_compound(members) -> bytes:
    """members: list of (name, offset, datatype bytes); version-1 compound."""
    size = 0
    body = b""
    for name, off, dt in members:
        body += _pad8(name.encode() + b"\0")
        body += struct.pack("<IB3xI4x4I", off, 0, 0, 0, 0, 0, 0)
        body += dt
        msize = struct.unpack_from("<I", dt, 4)[0]
        size = max(size, off + msize)
    n = len(members)
    return struct.pack("<BBBBI", 0x16, n & 0xFF, (n >> 8) & 0xFF, 0, size) + body


def dataspace(shape) -> bytes:
    shape = tuple(int(s) for s in shape)
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", s) for s in shape)


# --------------------------------------------------------------------------
# Object model
# --------------------------------------------------------------------------
class _VlenRef:
    """A variable-length item placed in the global heap."""

    def __init__(self, kind, payload):
        self.kind = kind          # "str" or "refs"
        self.payload = payload    # bytes, or list of objects
        self.index = None


class Attribute:
    def __init__(self, name, kind, value):
        self.name = name
        self.kind = kind          # vlen_str | fixed_str | quantity | dimlist | reflist | float
        self.value = value
        self.vlens = []


class Node:
    def __init__(self, name):
        self.name = name
        self.attrs: "OrderedDict[str, Attribute]" = OrderedDict()
        self.addr = None

    def set_attr(self, name, kind, value):
        self.attrs[name] = Attribute(name, kind, value)


class Group(Node):
    def __init__(self, name=""):
        super().__init__(name)
        self.children: "OrderedDict[str, Node]" = OrderedDict()
        self.btree_addr = self.snod_addr = self.heap_addr = self.heapdata_addr = None

    def group(self, name) -> "Group":
        if name not in self.children:
            self.children[name] = Group(name)
        return self.children[name]

    def dataset(self, name, data, units=None) -> "Dataset":
        d = Dataset(name, data)
        if units is not None:
            d.set_attr("units", "vlen_str", units)
        self.children[name] = d
        return d


class Dataset(Node):
    def __init__(self, name, data):
        super().__init__(name)
        data = np.ascontiguousarray(data)
        if data.dtype not in (np.float32, np.float64, np.int32):
            data = data.astype(np.float64)
        self.data = data
        self.data_addr = None
        self.scales = []          # (dim, Dataset) attached as dimension scales
        self.referrers = []       # (Dataset, dim) that use this one as a scale

    def attach_scale(self, dim: int, scale: "Dataset"):
        self.scales.append((dim, scale))
        scale.referrers.append((self, dim))


class MatFile:
    """An HDF5 file being assembled in memory."""

    def __init__(self):
        self.root = Group("")

    # Nebula properties ---------------------------------------------------
    def set_property_string(self, name, text):
        self.root.set_attr(name, "vlen_str", text)

    def set_property_quantity(self, name, value, unit):
        self.root.set_attr(name, "quantity", (float(value), unit))

    def group(self, path: str) -> Group:
        g = self.root
        for part in [p for p in path.split("/") if p]:
            g = g.group(part)
        return g

    # Serialisation --------------------------------------------------------
    def write(self, filename: str):
        with open(filename, "wb") as f:
            f.write(self.tobytes())

    def tobytes(self) -> bytes:
        groups, datasets = [], []

        def walk(g: Group):
            groups.append(g)
            for name, c in g.children.items():
                if isinstance(c, Group):
                    walk(c)
                else:
                    datasets.append(c)
        walk(self.root)

        # Finalise dimension-scale attributes.
        for d in datasets:
            if d.scales:
                rank = d.data.ndim
                per_dim = [[] for _ in range(rank)]
                for dim, s in d.scales:
                    per_dim[dim].append(s)
                d.set_attr("DIMENSION_LIST", "dimlist", per_dim)
            if d.referrers:
                d.set_attr("CLASS", "fixed_str", "DIMENSION_SCALE")
                d.set_attr("REFERENCE_LIST", "reflist", list(d.referrers))

        # Collect variable-length heap objects.
        vlens = []

        def add_vlen(kind, payload):
            v = _VlenRef(kind, payload)
            v.index = len(vlens) + 1
            vlens.append(v)
            return v

        for node in groups + datasets:
            for a in node.attrs.values():
                a.vlens = []
                if a.kind == "vlen_str":
                    a.vlens.append(add_vlen("str", a.value.encode()))
                elif a.kind == "quantity":
                    a.vlens.append(add_vlen("str", a.value[1].encode()))
                elif a.kind == "dimlist":
                    for lst in a.value:
                        a.vlens.append(add_vlen("refs", lst))

        # Layout pass: every block size is independent of the addresses.
        addr = 96

        def alloc(size):
            nonlocal addr
            a = addr
            addr += size + ((-size) % 8)
            return a

        for g in groups:
            g.addr = alloc(len(self._group_header(g, 0)))
            g.btree_addr = alloc(self._btree_size())
            g.snod_addr = alloc(self._snod_size())
            g.heap_addr = alloc(32)
            names, _ = self._heap_names(g)
            g.heapdata_addr = alloc(len(names))
        for d in datasets:
            d.addr = alloc(len(self._dataset_header(d, 0, 0)))
            d.data_addr = alloc(d.data.nbytes)
        gcol_payload = self._gcol(vlens, 0)
        gcol_addr = alloc(len(gcol_payload))
        eof = addr

        # Serialise pass.
        buf = bytearray(eof)
        buf[0:96] = self._superblock(eof)
        for g in groups:
            blob = self._group_header(g, gcol_addr)
            buf[g.addr:g.addr + len(blob)] = blob
            blob = self._btree(g)
            buf[g.btree_addr:g.btree_addr + len(blob)] = blob
            blob = self._snod(g)
            buf[g.snod_addr:g.snod_addr + len(blob)] = blob
            names, _ = self._heap_names(g)
            hdr = b"HEAP" + struct.pack("<B3xQQQ", 0, len(names), self._heap_free_offset(g), g.heapdata_addr)
            buf[g.heap_addr:g.heap_addr + 32] = hdr
            buf[g.heapdata_addr:g.heapdata_addr + len(names)] = names
        for d in datasets:
            blob = self._dataset_header(d, gcol_addr, d.data_addr)
            buf[d.addr:d.addr + len(blob)] = blob
            raw = d.data.astype(d.data.dtype.newbyteorder("<")).tobytes()
            buf[d.data_addr:d.data_addr + len(raw)] = raw
        blob = self._gcol(vlens, gcol_addr)
        buf[gcol_addr:gcol_addr + len(blob)] = blob
        return bytes(buf)

    # ---------------------------------------------------------------------
    def _superblock(self, eof):
        r = self.root
        sb = SIGNATURE
        sb += struct.pack("<8B", 0, 0, 0, 0, 0, 8, 8, 0)
        sb += struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQII", 0, r.addr, 1, 0) + struct.pack("<QQ", r.btree_addr, r.heap_addr)
        assert len(sb) == 96
        return sb

    @staticmethod
    def _object_header(messages):
        body = b""
        for mtype, flags, data in messages:
            data = _pad8(data)
            body += struct.pack("<HHB3x", mtype, len(data), flags) + data
        return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body

    def _attr_messages(self, node, gcol_addr):
        msgs = []
        for a in node.attrs.values():
            dt, ds, data = self._attr_encode(a, gcol_addr)
            name = a.name.encode() + b"\0"
            body = struct.pack("<BBHHH", 1, 0, len(name), len(dt), len(ds))
            body += _pad8(name) + _pad8(dt) + _pad8(ds) + data
            msgs.append((0x000C, 0, body))
        return msgs

    @staticmethod
    def _vlen_desc(length, gcol_addr, index):
        return struct.pack("<IQI", length, gcol_addr, index)

    def _attr_encode(self, a: Attribute, gcol_addr):
        if a.kind == "vlen_str":
            v = a.vlens[0]
            return dt_vlen_string(), dataspace(()), self._vlen_desc(len(v.payload), gcol_addr, v.index)
        if a.kind == "fixed_str":
            s = a.value.encode() + b"\0"
            return dt_fixed_string(len(s)), dataspace(()), s
        if a.kind == "quantity":
            v = a.vlens[0]
            dt = dt_compound([("value", 0, dt_float(8)), ("unit", 8, dt_vlen_string())])
            return dt, dataspace(()), struct.pack("<d", a.value[0]) + self._vlen_desc(len(v.payload), gcol_addr, v.index)
        if a.kind == "float":
            return dt_float(8), dataspace(()), struct.pack("<d", float(a.value))
        if a.kind == "dimlist":
            data = b"".join(self._vlen_desc(len(v.payload), gcol_addr, v.index) for v in a.vlens)
            return dt_vlen_sequence(dt_objref()), dataspace((len(a.vlens),)), data
        if a.kind == "reflist":
            dt = dt_compound([("dataset", 0, dt_objref()), ("dimension", 8, dt_int(4, True))])
            data = b"".join(struct.pack("<Qi", (ds.addr or 0), dim) for ds, dim in a.value)
            return dt, dataspace((len(a.value),)), data
        raise ValueError(a.kind)

    def _group_header(self, g: Group, gcol_addr):
        msgs = [(0x0011, 0, struct.pack("<QQ", g.btree_addr or 0, g.heap_addr or 0))]
        msgs += self._attr_messages(g, gcol_addr)
        return self._object_header(msgs)

    def _dataset_header(self, d: Dataset, gcol_addr, data_addr):
        if d.data.dtype == np.float32:
            dt = dt_float(4)
        elif d.data.dtype == np.float64:
            dt = dt_float(8)
        else:
            dt = dt_int(4, True)
        msgs = [
            (0x0001, 0, dataspace(d.data.shape)),
            (0x0003, 1, dt),
            (0x0005, 1, struct.pack("<BBBB", 2, 2, 2, 0)),
            (0x0008, 0, struct.pack("<BBQQ", 3, 1, data_addr, d.data.nbytes)),
        ]
        msgs += self._attr_messages(d, gcol_addr)
        return self._object_header(msgs)

    @staticmethod
    def _btree_size():
        return 24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8

    @staticmethod
    def _snod_size():
        return 8 + 2 * LEAF_K * 40

    @staticmethod
    def _sorted_children(g: Group):
        return sorted(g.children.items(), key=lambda kv: kv[0].encode())

    def _heap_names(self, g: Group):
        data = _pad8(b"\0")
        offsets = {}
        for name, _ in self._sorted_children(g):
            offsets[name] = len(data)
            data += _pad8(name.encode() + b"\0")
        free_off = len(data)
        data += struct.pack("<QQ", HEAP_FREE_NULL, 16)
        return data, (offsets, free_off)

    def _heap_free_offset(self, g):
        return self._heap_names(g)[1][1]

    def _btree(self, g: Group):
        children = self._sorted_children(g)
        assert len(children) <= 2 * LEAF_K, "group too large for one symbol table node"
        _, (offsets, _) = self._heap_names(g)
        last = offsets[children[-1][0]] if children else 0
        b = b"TREE" + struct.pack("<BBH", 0, 0, 1) + struct.pack("<QQ", UNDEF, UNDEF)
        b += struct.pack("<QQQ", 0, g.snod_addr, last)
        return b + b"\0" * (self._btree_size() - len(b))

    def _snod(self, g: Group):
        children = self._sorted_children(g)
        _, (offsets, _) = self._heap_names(g)
        b = b"SNOD" + struct.pack("<BBH", 1, 0, len(children))
        for name, c in children:
            if isinstance(c, Group):
                b += struct.pack("<QQII", offsets[name], c.addr, 1, 0) + struct.pack("<QQ", c.btree_addr, c.heap_addr)
            else:
                b += struct.pack("<QQII", offsets[name], c.addr, 0, 0) + b"\0" * 16
        return b + b"\0" * (self._snod_size() - len(b))

    def _gcol(self, vlens, gcol_addr):
        body = b""
        for v in vlens:
            if v.kind == "str":
                payload = v.payload
            else:
                payload = b"".join(struct.pack("<Q", (o.addr or 0)) for o in v.payload)
            body += struct.pack("<HHIQ", v.index, 1, 0, len(payload)) + _pad8(payload)
        size = 16 + len(body)
        total = max(GCOL_MIN, size + 16)
        free = total - size
        body += struct.pack("<HHIQ", 0, 0, 0, free) + b"\0" * (free - 16)
        return b"GCOL" + struct.pack("<B3xQ", 1, total) + body
