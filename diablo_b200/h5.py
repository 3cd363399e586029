"""HDF5 files without an HDF5 library: a writer and a reader for the subset
that DIABLO's output files use.

The reference writes mean.h5 / tke.h5 / stats.h5 (WriteStatH5,
for/hdf5.f:1466-1622) and start.h5 / out.h5 / end.h5 (WriteHDF5,
for/hdf5.f:5-295) through the HDF5 library.  This image has none, so this
module writes the format itself, in the layout of the HDF5 1.8 library with
its default (earliest) format versions, as the reference's own files have
(KH_test/grid.h5 is one): superblock version 0 with 8-byte offsets and
lengths, version-1 object headers, groups as symbol tables (a version-1
B-tree, its symbol-table nodes and a local heap of names), contiguous
datasets, version-1 attribute messages.

Supported types: little-endian IEEE float64 / float32, signed int32 / int64
and fixed-length ASCII strings; dataspaces scalar or simple of any rank.
The writer builds a whole file at once (`write(path, root)`); a caller that
appends (the statistics files, one group entry per SAVE_STATS call) reads the
tree back, extends it and writes it again.  The reader also follows object
header continuation messages and B-trees of several levels, so it reads files
that the HDF5 library wrote with these versions.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
_SIG = b"\x89HDF\r\n\x1a\n"


@dataclass
class Dataset:
    data: np.ndarray
    attrs: dict = field(default_factory=dict)


@dataclass
class Group:
    children: dict = field(default_factory=dict)      # name -> Group | Dataset, any order
    attrs: dict = field(default_factory=dict)

    def group(self, name: str) -> "Group":
        """The child group `name`, created when missing."""
        g = self.children.get(name)
        if g is None:
            g = self.children[name] = Group()
        if not isinstance(g, Group):
            raise TypeError(f"{name} is a dataset, not a group")
        return g


# --- encoding -------------------------------------------------------------------
def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


def _as_array(value) -> np.ndarray:
    if isinstance(value, (str, bytes)):
        s = value.encode("ascii") if isinstance(value, str) else value
        return np.array(s, dtype=f"S{max(len(s), 1)}")
    a = np.asarray(value)
    if a.dtype.kind == "U":
        a = a.astype("S")
    if a.dtype.kind == "f":
        a = a.astype("<f8" if a.dtype.itemsize == 8 else "<f4")
    elif a.dtype.kind in "iu":
        a = a.astype("<i8" if a.dtype.itemsize == 8 else "<i4")
    elif a.dtype.kind == "b":
        a = a.astype("<i4")
    elif a.dtype.kind != "S":
        raise TypeError(f"unsupported dtype {a.dtype}")
    return np.require(a, requirements="C")          # keeps rank 0 (a scalar dataspace)


def _datatype(a: np.ndarray) -> bytes:
    """Datatype message (version 1)."""
    k, n = a.dtype.kind, a.dtype.itemsize
    if k == "f":
        if n == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            bits = bytes([0x20, 63, 0])
        else:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            bits = bytes([0x20, 31, 0])
        return bytes([0x11]) + bits + struct.pack("<I", n) + props
    if k == "i":
        return bytes([0x10, 0x08, 0, 0]) + struct.pack("<I", n) + struct.pack("<HH", 0, 8 * n)
    if k == "S":
        return bytes([0x13, 0x00, 0, 0]) + struct.pack("<I", n)     # null-terminated ASCII
    raise TypeError(a.dtype)


def _dataspace(a: np.ndarray) -> bytes:
    """Dataspace message (version 1); rank 0 is a scalar."""
    return struct.pack("<BBBBI", 1, a.ndim, 0, 0, 0) + b"".join(struct.pack("<Q", d) for d in a.shape)


def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _attribute(name: str, value) -> bytes:
    a = _as_array(value)
    nm = name.encode("ascii") + b"\0"
    dt, ds = _datatype(a), _dataspace(a)
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(ds)) + _pad8(nm) + _pad8(dt) + _pad8(ds) + a.tobytes()
    return _message(0x000C, body)


def _object_header(messages: list[bytes]) -> bytes:
    body = b"".join(messages)
    return struct.pack("<BBHII", 1, 0, len(messages), 1, len(body)) + b"\0" * 4 + body


def write(path: str, root: Group) -> None:
    """Write the tree `root` as an HDF5 file."""
    out = bytearray()

    def groups_of(g: Group):
        yield g
        for c in g.children.values():
            if isinstance(c, Group):
                yield from groups_of(c)

    # symbol-table nodes hold 2K entries: K large enough for the biggest group
    leaf_k = max(4, (max(len(g.children) for g in groups_of(root)) + 1) // 2)
    if leaf_k > 0xFFFF:
        raise ValueError("too many members in one group")
    internal_k = 16
    out += b"\0" * 96                               # superblock, filled in at the end

    def alloc(n: int) -> int:
        addr = len(out)
        out.extend(b"\0" * n)
        return addr

    def put(addr: int, b: bytes) -> None:
        out[addr:addr + len(b)] = b

    def emit_dataset(d: Dataset) -> int:
        a = _as_array(d.data)
        daddr = alloc(len(_pad8(a.tobytes()))) if a.nbytes else UNDEF
        if a.nbytes:
            put(daddr, a.tobytes())
        msgs = [_message(0x0001, _dataspace(a)), _message(0x0003, _datatype(a), flags=1),
                _message(0x0005, bytes([2, 2, 2, 0])),                        # fill value: none defined
                _message(0x0008, struct.pack("<BBQQ", 3, 1, daddr, a.nbytes))]  # contiguous layout
        msgs += [_attribute(k, v) for k, v in d.attrs.items()]
        oh = _object_header(msgs)
        addr = alloc(len(oh))
        put(addr, oh)
        return addr

    def emit_group(g: Group) -> tuple[int, int, int]:
        """Returns (object header address, B-tree address, heap address)."""
        names = sorted(g.children)
        entries = []
        for nm in names:
            c = g.children[nm]
            if isinstance(c, Group):
                oh, bt, hp = emit_group(c)
                entries.append((nm, oh, 1, struct.pack("<QQ", bt, hp)))
            else:
                entries.append((nm, emit_dataset(c), 0, b"\0" * 16))
        # local heap: the empty string at offset 0, then every name
        heap = bytearray(b"\0" * 8)
        offsets = {}
        for nm in names:
            offsets[nm] = len(heap)
            heap += _pad8(nm.encode("ascii") + b"\0")
        heap_data = alloc(len(heap))
        put(heap_data, bytes(heap))
        heap_addr = alloc(32)
        put(heap_addr, b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), UNDEF, heap_data))
        # one symbol-table node with every entry, in name order
        snod = bytearray(b"SNOD" + struct.pack("<BBH", 1, 0, len(entries)))
        for nm, oh, cache, scratch in entries:
            snod += struct.pack("<QQII", offsets[nm], oh, cache, 0) + scratch
        snod += b"\0" * (40 * (2 * leaf_k - len(entries)))
        snod_addr = alloc(len(snod))
        put(snod_addr, bytes(snod))
        # a one-node B-tree: key 0 (the empty name), child 0, key 1 (the last name)
        node = bytearray(b"TREE" + struct.pack("<BBHQQ", 0, 0, 1 if entries else 0, UNDEF, UNDEF))
        if entries:
            node += struct.pack("<QQQ", 0, snod_addr, offsets[names[-1]])
        node += b"\0" * (24 + (2 * internal_k + 1) * 8 + 2 * internal_k * 8 - len(node))
        bt_addr = alloc(len(node))
        put(bt_addr, bytes(node))
        msgs = [_message(0x0011, struct.pack("<QQ", bt_addr, heap_addr))]
        msgs += [_attribute(k, v) for k, v in g.attrs.items()]
        oh = _object_header(msgs)
        oh_addr = alloc(len(oh))
        put(oh_addr, oh)
        return oh_addr, bt_addr, heap_addr

    root_oh, root_bt, root_hp = emit_group(root)
    sb = _SIG + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, leaf_k, internal_k, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, len(out), UNDEF)
    sb += struct.pack("<QQII", 0, root_oh, 1, 0) + struct.pack("<QQ", root_bt, root_hp)
    assert len(sb) == 96
    put(0, sb)
    with open(path, "wb") as f:
        f.write(bytes(out))


# --- decoding -------------------------------------------------------------------
class _Reader:
    def __init__(self, buf: bytes):
        if buf[:8] != _SIG:
            raise ValueError("not an HDF5 file (signature)")
        if buf[8] != 0:
            raise ValueError(f"superblock version {buf[8]} is not supported (0 only)")
        if buf[13] != 8 or buf[14] != 8:
            raise ValueError("only 8-byte offsets and lengths are supported")
        self.b = buf
        root_oh = struct.unpack_from("<Q", buf, 56 + 8)[0]
        self.root = root_oh

    def _messages(self, addr: int):
        b = self.b
        ver, _, nmsg, _, size = struct.unpack_from("<BBHII", b, addr)
        if ver != 1:
            raise ValueError(f"object header version {ver} is not supported (1 only)")
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            pos, length = blocks.pop(0)
            end = pos + length
            while pos + 8 <= end and len(out) < nmsg:
                mtype, msize, flags = struct.unpack_from("<HHB", b, pos)
                body = b[pos + 8:pos + 8 + msize]
                pos += 8 + msize
                if mtype == 0x0010:                       # continuation
                    blocks.append(struct.unpack_from("<QQ", body, 0))
                out.append((mtype, body))
        return out

    @staticmethod
    def _dtype(body: bytes):
        cv = body[0]
        cls, ver = cv & 0x0F, cv >> 4
        size = struct.unpack_from("<I", body, 4)[0]
        bits = body[1]
        if cls == 1:
            return np.dtype(("<" if not (bits & 1) else ">") + f"f{size}")
        if cls == 0:
            signed = bool(bits & 0x08)
            return np.dtype(("<" if not (bits & 1) else ">") + ("i" if signed else "u") + str(size))
        if cls == 3:
            return np.dtype(f"S{size}")
        raise ValueError(f"datatype class {cls} (version {ver}) is not supported")

    @staticmethod
    def _shape(body: bytes):
        ver, rank, flags = body[0], body[1], body[2]
        off = 8 if ver == 1 else 4
        return tuple(struct.unpack_from("<Q", body, off + 8 * i)[0] for i in range(rank))

    def _attribute(self, body: bytes):
        ver = body[0]
        if ver != 1:
            raise ValueError(f"attribute message version {ver} is not supported (1 only)")
        nsz, dsz, ssz = struct.unpack_from("<HHH", body, 2)
        pos = 8
        name = body[pos:pos + nsz].split(b"\0")[0].decode("ascii")
        pos += nsz + (-nsz % 8)
        dt = self._dtype(body[pos:pos + dsz])
        pos += dsz + (-dsz % 8)
        shape = self._shape(body[pos:pos + ssz])
        pos += ssz + (-ssz % 8)
        n = int(np.prod(shape)) if shape else 1
        a = np.frombuffer(body, dtype=dt, count=n, offset=pos).reshape(shape).copy()
        return name, a

    def _btree_entries(self, bt_addr: int, heap_data: int):
        b = self.b
        if b[bt_addr:bt_addr + 4] != b"TREE":
            raise ValueError("bad B-tree signature")
        ntype, level, used = struct.unpack_from("<BBH", b, bt_addr + 4)
        pos = bt_addr + 24
        out = []
        for i in range(used):
            child = struct.unpack_from("<Q", b, pos + 8 + 16 * i)[0]
            if level > 0:
                out += self._btree_entries(child, heap_data)
            else:
                if b[child:child + 4] != b"SNOD":
                    raise ValueError("bad symbol-table node signature")
                nsym = struct.unpack_from("<H", b, child + 6)[0]
                for k in range(nsym):
                    e = child + 8 + 40 * k
                    name_off, oh, cache = struct.unpack_from("<QQI", b, e)
                    s = heap_data + name_off
                    name = b[s:b.index(b"\0", s)].decode("ascii")
                    out.append((name, oh))
        return out

    def node(self, addr: int):
        msgs = self._messages(addr)
        attrs = {}
        stab = shape = dt = layout = None
        for mtype, body in msgs:
            if mtype == 0x0011:
                stab = struct.unpack_from("<QQ", body, 0)
            elif mtype == 0x0001:
                shape = self._shape(body)
            elif mtype == 0x0003:
                dt = self._dtype(body)
            elif mtype == 0x0008:
                layout = body
            elif mtype == 0x000C:
                k, v = self._attribute(body)
                attrs[k] = v
        if stab is not None:
            bt, heap = stab
            if self.b[heap:heap + 4] != b"HEAP":
                raise ValueError("bad local heap signature")
            heap_data = struct.unpack_from("<Q", self.b, heap + 24)[0]
            g = Group(attrs=attrs)
            for name, oh in self._btree_entries(bt, heap_data):
                g.children[name] = self.node(oh)
            return g
        if layout is None or dt is None or shape is None:
            raise ValueError("object is neither a group nor a dataset this reader handles")
        ver, cls = layout[0], layout[1]
        n = int(np.prod(shape)) if shape else 1
        if ver == 3 and cls == 1:                         # contiguous
            daddr, size = struct.unpack_from("<QQ", layout, 2)
            data = (np.zeros(shape, dtype=dt) if daddr == UNDEF else
                    np.frombuffer(self.b, dtype=dt, count=n, offset=daddr).reshape(shape).copy())
        elif ver == 3 and cls == 0:                       # compact
            size = struct.unpack_from("<H", layout, 2)[0]
            data = np.frombuffer(layout, dtype=dt, count=n, offset=4).reshape(shape).copy()
        else:
            raise ValueError(f"data layout version {ver} class {cls} is not supported")
        return Dataset(data, attrs)


def read(path: str) -> Group:
    """The whole file as a tree of Group / Dataset."""
    with open(path, "rb") as f:
        r = _Reader(f.read())
    return r.node(r.root)


def is_hdf5(path: str) -> bool:
    with open(path, "rb") as f:
        return f.read(8) == _SIG
