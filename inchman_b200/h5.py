"""HDF5 files written and read without libhdf5.

The reference writes its results with libhdf5 (DiffusionModel.cpp:934-1296,
InchmanDiffusionModel.cpp:240-274; layout in doc/source/hdf5.rst) and its analysis
scripts read them with h5py (python/gpgmp/io.py:189-290).  Neither library is in this
image, so this module writes the subset of the format those files use, following the
published HDF5 file format specification in its earliest layout -- the one libhdf5
itself writes by default:

  superblock version 0 (8-byte offsets and lengths), version 1 object headers,
  groups as symbol tables (a local heap of names, a version 1 B-tree of symbol table
  nodes, names sorted), contiguous datasets, version 1 attribute messages, datatypes
  32/64-bit little-endian integers and IEEE floats, fixed-length and variable-length
  (global heap) ASCII strings.

`read` parses the same subset (plus layout message versions 1-2 and object header
continuations) and is what the tests check the writer with; it also reads files that
libhdf5 wrote in this layout.
"""
from __future__ import annotations

import struct
from typing import Dict, List, Optional, Union

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K = 4          # symbol table node holds up to 2 LEAF_K names (libhdf5's default)
NODE_K = 16         # B-tree node holds up to 2 NODE_K children (libhdf5's default)
HEAP_FREE_NULL = 1  # "no next free block" in a local heap's free list

# object header message types
MSG_NIL, MSG_DATASPACE, MSG_DATATYPE, MSG_FILL, MSG_LAYOUT = 0x0, 0x1, 0x3, 0x5, 0x8
MSG_ATTRIBUTE, MSG_CONTINUATION, MSG_SYMBOL_TABLE = 0xC, 0x10, 0x11


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


def _align8(n: int) -> int:
    return (n + 7) & ~7


# ---- datatypes -----------------------------------------------------------------

def _dt_int(size: int, signed: bool) -> bytes:
    return struct.pack("<B3BI", 0x10, 0x08 if signed else 0, 0, 0, size) + struct.pack("<HH", 0, 8 * size)


def _dt_float(size: int) -> bytes:
    if size == 4:
        return struct.pack("<B3BI", 0x11, 0x20, 31, 0, 4) + struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
    return struct.pack("<B3BI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)


def _dt_fixed_string(n: int) -> bytes:
    return struct.pack("<B3BI", 0x13, 0, 0, 0, n)          # null-terminated ASCII


def _dt_vlen_string() -> bytes:
    # sequence length (4) + global heap collection address (8) + object index (4);
    # the base type is an unsigned byte
    return struct.pack("<B3BI", 0x19, 0x01, 0, 0, 16) + _dt_int(1, False)


def _dt_numpy(dt: np.dtype) -> bytes:
    dt = np.dtype(dt)
    if dt.byteorder == ">":
        raise ValueError("big-endian data")
    if dt.kind in "iu" and dt.itemsize in (1, 2, 4, 8):
        return _dt_int(dt.itemsize, dt.kind == "i")
    if dt.kind == "f" and dt.itemsize in (4, 8):
        return _dt_float(dt.itemsize)
    raise ValueError(f"unsupported dtype {dt}")


def _dataspace(shape) -> bytes:
    return struct.pack("<BBBBI", 1, len(shape), 0, 0, 0) + b"".join(struct.pack("<Q", int(d)) for d in shape)


# ---- messages and object headers ------------------------------------------------

def _msg(mtype: int, data: bytes, flags: int = 0) -> bytes:
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _ohdr(msgs: List[bytes]) -> bytes:
    body = b"".join(msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


def _attr_msg(name: str, value) -> bytes:
    if isinstance(value, str):
        raw = value.encode("ascii") + b"\0"
        dt, space, data = _dt_fixed_string(len(raw)), struct.pack("<BBBBI", 1, 0, 0, 0, 0), raw
    else:
        a = np.ascontiguousarray(value)
        if a.ndim == 0:
            a = a.reshape(1)
        dt, space, data = _dt_numpy(a.dtype), _dataspace(a.shape), a.tobytes()
    nm = name.encode("ascii") + b"\0"
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(space)) + _pad8(nm) + _pad8(dt) + _pad8(space) + data
    return _msg(MSG_ATTRIBUTE, body)


FILL_DEFAULT = bytes([1, 2, 2, 1, 0, 0, 0, 0])   # version 1: late allocation, fill if set, default value


# ---- the object tree ------------------------------------------------------------

class Dataset:
    """A contiguous dataset: a numpy array, a list of strings (variable-length ASCII),
    or one string (scalar, fixed length, null-terminated)."""

    def __init__(self, data: Union[np.ndarray, List[str], str]):
        self.attrs: Dict[str, object] = {}
        self.data = data

    def _encode(self, gheap_addr: int):
        d = self.data
        if isinstance(d, str):
            raw = d.encode("ascii") + b"\0"
            return _dt_fixed_string(len(raw)), struct.pack("<BBBBI", 1, 0, 0, 0, 0), raw
        if isinstance(d, list):
            raw = b"".join(struct.pack("<IQI", len(s.encode("ascii")), gheap_addr, i + 1) for i, s in enumerate(d))
            return _dt_vlen_string(), _dataspace((len(d),)), raw
        a = np.ascontiguousarray(d)
        return _dt_numpy(a.dtype), _dataspace(a.shape), a

    def raw_size(self) -> int:
        d = self.data
        if isinstance(d, str):
            return len(d.encode("ascii")) + 1
        if isinstance(d, list):
            return 16 * len(d)
        return int(np.asarray(d).nbytes)


class Group:
    def __init__(self):
        self.attrs: Dict[str, object] = {}
        self.children: Dict[str, Union["Group", Dataset]] = {}

    def create_group(self, name: str) -> "Group":
        if name in self.children:
            raise ValueError(f"{name!r} exists")
        g = Group()
        self.children[name] = g
        return g

    def require_group(self, name: str) -> "Group":
        g = self.children.get(name)
        return g if isinstance(g, Group) else self.create_group(name)

    def create_dataset(self, name: str, data) -> Dataset:
        if name in self.children:
            raise ValueError(f"{name!r} exists")
        d = Dataset(data)
        self.children[name] = d
        return d

    def __contains__(self, name):
        return name in self.children

    def __getitem__(self, name):
        return self.children[name]


# ---- layout and writing ---------------------------------------------------------

class _Writer:
    def __init__(self):
        self.cursor = 0
        self.blocks = []     # (address, bytes or callable -> bytes)

    def alloc(self, size: int) -> int:
        a = self.cursor
        self.cursor = _align8(self.cursor + size)
        return a


def _group_plan(w: _Writer, g: Group, plan: dict):
    """Assigns the addresses of g's header, heap, nodes and (recursively) children."""
    names = sorted(g.children, key=lambda s: s.encode("ascii"))
    oh_msgs = [_msg(MSG_SYMBOL_TABLE, struct.pack("<QQ", 0, 0), 1)] + [_attr_msg(k, v) for k, v in g.attrs.items()]
    p = {"names": names}
    p["oh"] = w.alloc(len(_ohdr(oh_msgs)))
    # local heap: "" at 0, then the names, then one free block
    offs, seg = {}, bytearray(8)
    for nm in names:
        offs[nm] = len(seg)
        seg += _pad8(nm.encode("ascii") + b"\0")
    p["free_off"] = len(seg)
    seg += struct.pack("<QQ", HEAP_FREE_NULL, 16)
    p["heap_seg"], p["name_off"] = bytes(seg), offs
    p["heap"] = w.alloc(32)
    p["heap_data"] = w.alloc(len(seg))
    # symbol table nodes: names in order, 2 LEAF_K per node
    per = 2 * LEAF_K
    chunks = [names[i:i + per] for i in range(0, len(names), per)]
    p["snods"] = [(w.alloc(8 + per * 40), c) for c in chunks]
    # B-tree: level 0 points at the symbol table nodes; upper levels until one root
    level_items = [(a, c[-1]) for a, c in p["snods"]]        # (child address, last name in the subtree)
    levels = []
    lvl = 0
    while True:
        nodes = []
        groups_ = [level_items[i:i + 2 * NODE_K] for i in range(0, len(level_items), 2 * NODE_K)] or [[]]
        for items in groups_:
            nodes.append({"addr": w.alloc(24 + (2 * NODE_K + 1) * 8 + 2 * NODE_K * 8), "items": items, "level": lvl})
        levels.append(nodes)
        if len(nodes) == 1:
            break
        level_items = [(n["addr"], n["items"][-1][1]) for n in nodes]
        lvl += 1
    p["btree_levels"] = levels
    p["btree"] = levels[-1][0]["addr"]
    plan[id(g)] = p
    for nm in names:
        c = g.children[nm]
        if isinstance(c, Group):
            _group_plan(w, c, plan)
        else:
            _dataset_plan(w, c, plan)


def _dataset_plan(w: _Writer, d: Dataset, plan: dict):
    p = {}
    dt, space, _ = d._encode(0)
    msgs = [_msg(MSG_DATASPACE, space), _msg(MSG_DATATYPE, dt, 1), _msg(MSG_FILL, FILL_DEFAULT, 1),
            _msg(MSG_LAYOUT, struct.pack("<BBQQ", 3, 1, 0, 0))] + [_attr_msg(k, v) for k, v in d.attrs.items()]
    p["oh"] = w.alloc(len(_ohdr(msgs)))
    p["raw"] = w.alloc(d.raw_size()) if d.raw_size() else UNDEF
    if isinstance(d.data, list):
        objs = b""
        for s in d.data:
            b = s.encode("ascii")
            objs += struct.pack("<HH4xQ", 0, 0, len(b)) + _pad8(b)   # index filled in when written
        size = max(4096, 16 + len(objs) + 16)
        p["gcol_size"] = size
        p["gcol"] = w.alloc(size)
    plan[id(d)] = p


def _emit_group(g: Group, plan: dict, out: dict):
    p = plan[id(g)]
    msgs = [_msg(MSG_SYMBOL_TABLE, struct.pack("<QQ", p["btree"], p["heap"]), 1)] + \
           [_attr_msg(k, v) for k, v in g.attrs.items()]
    out[p["oh"]] = _ohdr(msgs)
    seg = p["heap_seg"]
    out[p["heap"]] = b"HEAP" + struct.pack("<B3xQQQ", 0, len(seg), p["free_off"], p["heap_data"])
    out[p["heap_data"]] = seg
    per = 2 * LEAF_K
    for addr, names in p["snods"]:
        body = b"SNOD" + struct.pack("<BBH", 1, 0, len(names))
        for nm in names:
            child = plan[id(g.children[nm])]
            body += struct.pack("<QQII16x", p["name_off"][nm], child["oh"], 0, 0)
        out[addr] = body + b"\0" * (8 + per * 40 - len(body))
    full = 24 + (2 * NODE_K + 1) * 8 + 2 * NODE_K * 8
    for nodes in p["btree_levels"]:
        for i, n in enumerate(nodes):
            left = nodes[i - 1]["addr"] if i > 0 else UNDEF
            right = nodes[i + 1]["addr"] if i + 1 < len(nodes) else UNDEF
            # left key of the node: the last name of the previous node (or "")
            k0 = p["name_off"][nodes[i - 1]["items"][-1][1]] if i > 0 else 0
            body = b"TREE" + struct.pack("<BBHQQ", 0, n["level"], len(n["items"]), left, right)
            body += struct.pack("<Q", k0)
            for child, last in n["items"]:
                body += struct.pack("<QQ", child, p["name_off"][last])
            out[n["addr"]] = body + b"\0" * (full - len(body))
    for nm in p["names"]:
        c = g.children[nm]
        if isinstance(c, Group):
            _emit_group(c, plan, out)
        else:
            _emit_dataset(c, plan, out)


def _emit_dataset(d: Dataset, plan: dict, out: dict):
    p = plan[id(d)]
    dt, space, raw = d._encode(p.get("gcol", 0))
    layout = struct.pack("<BBQQ", 3, 1, p["raw"], d.raw_size())
    msgs = [_msg(MSG_DATASPACE, space), _msg(MSG_DATATYPE, dt, 1), _msg(MSG_FILL, FILL_DEFAULT, 1),
            _msg(MSG_LAYOUT, layout)] + [_attr_msg(k, v) for k, v in d.attrs.items()]
    out[p["oh"]] = _ohdr(msgs)
    if p["raw"] != UNDEF:
        out[p["raw"]] = raw
    if "gcol" in p:
        body = b"GCOL" + struct.pack("<B3xQ", 1, p["gcol_size"])
        for i, s in enumerate(d.data):
            b = s.encode("ascii")
            body += struct.pack("<HH4xQ", i + 1, 0, len(b)) + _pad8(b)
        free = p["gcol_size"] - len(body)
        body += struct.pack("<HH4xQ", 0, 0, free)
        out[p["gcol"]] = body + b"\0" * (p["gcol_size"] - len(body))


def write(path: str, root: Group):
    """Writes the tree under root to path (overwriting it)."""
    w = _Writer()
    sb_size = 8 + 8 + 4 + 4 + 4 * 8 + 40
    w.alloc(sb_size)
    plan: dict = {}
    _group_plan(w, root, plan)
    out: dict = {}
    _emit_group(root, plan, out)
    eof = w.cursor
    rp = plan[id(root)]
    sb = SIGNATURE + struct.pack("<BBBBBBBB", 0, 0, 0, 0, 0, 8, 8, 0) + struct.pack("<HHI", LEAF_K, NODE_K, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    sb += struct.pack("<QQII", 0, rp["oh"], 1, 0) + struct.pack("<QQ", rp["btree"], rp["heap"])
    out[0] = sb
    with open(path, "wb") as f:
        pos = 0
        for addr in sorted(out):
            if addr > pos:
                f.write(b"\0" * (addr - pos))
                pos = addr
            data = out[addr]
            if isinstance(data, np.ndarray):
                data.tofile(f)
                pos += data.nbytes
            else:
                f.write(data)
                pos += len(data)
        if eof > pos:
            f.write(b"\0" * (eof - pos))


# ---- reading --------------------------------------------------------------------

class Node:
    """A group (children) or dataset (value) read back, with its attributes."""

    def __init__(self, kind: str):
        self.kind = kind
        self.attrs: Dict[str, object] = {}
        self.children: Dict[str, "Node"] = {}
        self.value = None

    def __getitem__(self, path: str) -> "Node":
        n = self
        for part in path.strip("/").split("/"):
            if part:
                n = n.children[part]
        return n

    def __contains__(self, name):
        return name in self.children

    def __iter__(self):
        return iter(self.children)      # names in the file's (sorted) order


class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        for off in [0] + [512 << i for i in range(16)]:
            if off + 8 <= len(data) and data[off:off + 8] == SIGNATURE:
                break
        else:
            raise ValueError("not an HDF5 file")
        sb = off
        ver = data[sb + 8]
        if ver not in (0, 1):
            raise ValueError(f"superblock version {ver} not supported")
        if data[sb + 13] != 8 or data[sb + 14] != 8:
            raise ValueError("only 8-byte offsets and lengths are supported")
        self.leaf_k, self.node_k = struct.unpack_from("<HH", data, sb + 16)
        p = sb + 24 + (4 if ver == 1 else 0)
        self.base, _, self.eof, _ = struct.unpack_from("<QQQQ", data, p)
        self.root_entry = p + 32

    def u(self, fmt, addr):
        return struct.unpack_from(fmt, self.d, self.base + addr)

    def messages(self, oh: int):
        version = self.d[self.base + oh]
        if version != 1:
            raise ValueError(f"object header version {version} not supported")
        nmsg, _, size = self.u("<HII", oh + 2)
        chunks, out = [(oh + 16, size)], []
        while chunks and len(out) < nmsg:
            a, n = chunks.pop(0)
            p = a
            while p + 8 <= a + n and len(out) < nmsg:
                t, s, flags = self.u("<HHB", p)
                body = self.d[self.base + p + 8:self.base + p + 8 + s]
                if t == MSG_CONTINUATION:
                    chunks.append(struct.unpack_from("<QQ", body))
                out.append((t, body))
                p += 8 + s
        return out

    def datatype(self, b: bytes):
        cv = b[0]
        cls, ver = cv & 0x0F, cv >> 4
        bits = b[1] | (b[2] << 8) | (b[3] << 16)
        size = struct.unpack_from("<I", b, 4)[0]
        if cls == 0:
            if bits & 1:
                raise ValueError("big-endian integers")
            return ("int", np.dtype(("i" if bits & 8 else "u") + str(size)).newbyteorder("<"))
        if cls == 1:
            if bits & 1:
                raise ValueError("big-endian floats")
            return ("float", np.dtype("<f" + str(size)))
        if cls == 3:
            return ("string", size)
        if cls == 9 and (bits & 0x0F) == 1:
            return ("vlen_string", size)
        raise ValueError(f"datatype class {cls} not supported")

    def dataspace(self, b: bytes):
        ver, rank, flags = b[0], b[1], b[2]
        p = 8 if ver == 1 else 4
        if ver == 2 and b[3] == 0:
            return ()
        return tuple(struct.unpack_from("<Q", b, p + 8 * i)[0] for i in range(rank))

    def vlen_string(self, rec: bytes) -> str:
        n, col, idx = struct.unpack("<IQI", rec)
        if n == 0:
            return ""
        if self.d[self.base + col:self.base + col + 4] != b"GCOL":
            raise ValueError("bad global heap collection")
        size = self.u("<Q", col + 8)[0]
        p = col + 16
        while p + 16 <= col + size:
            i, _, osz = self.u("<HH4xQ", p)
            if i == 0:
                break
            if i == idx:
                return self.d[self.base + p + 16:self.base + p + 16 + n].decode("ascii")
            p += 16 + _align8(osz)
        raise ValueError(f"global heap object {idx} not found")

    def values(self, dt, shape, raw: bytes):
        kind = dt[0]
        if kind in ("int", "float"):
            return np.frombuffer(raw, dtype=dt[1], count=int(np.prod(shape)) if shape else 1).reshape(shape)
        if kind == "string":
            n = dt[1]
            vals = [raw[i * n:(i + 1) * n].split(b"\0")[0].decode("ascii") for i in range(max(1, int(np.prod(shape))))]
            return vals[0] if shape == () else vals
        vals = [self.vlen_string(raw[i * 16:(i + 1) * 16]) for i in range(int(np.prod(shape)) if shape else 1)]
        return vals[0] if shape == () else vals

    def obj(self, oh: int) -> Node:
        msgs = self.messages(oh)
        types = [t for t, _ in msgs]
        node = Node("group" if MSG_SYMBOL_TABLE in types else "dataset")
        dt = shape = None
        for t, b in msgs:
            if t == MSG_ATTRIBUTE:
                ver = b[0]
                if ver != 1:
                    raise ValueError(f"attribute message version {ver} not supported")
                nsz, tsz, ssz = struct.unpack_from("<HHH", b, 2)
                p = 8
                name = b[p:p + nsz].split(b"\0")[0].decode("ascii")
                p += _align8(nsz)
                adt = self.datatype(b[p:p + tsz])
                p += _align8(tsz)
                ash = self.dataspace(b[p:p + ssz])
                p += _align8(ssz)
                node.attrs[name] = self.values(adt, ash, b[p:])
            elif t == MSG_DATATYPE:
                dt = self.datatype(b)
            elif t == MSG_DATASPACE:
                shape = self.dataspace(b)
            elif t == MSG_SYMBOL_TABLE:
                bt, heap = struct.unpack_from("<QQ", b)
                for name, child in self.group_entries(bt, heap):
                    node.children[name] = self.obj(child)
        if node.kind == "dataset":
            raw = self.raw(msgs, dt, shape)
            node.value = self.values(dt, shape, raw)
        return node

    def raw(self, msgs, dt, shape) -> bytes:
        for t, b in msgs:
            if t != MSG_LAYOUT:
                continue
            ver = b[0]
            if ver == 3:
                cls = b[1]
                if cls == 1:
                    addr, size = struct.unpack_from("<QQ", b, 2)
                    return b"" if addr == UNDEF else self.d[self.base + addr:self.base + addr + size]
                if cls == 0:
                    size = struct.unpack_from("<H", b, 2)[0]
                    return b[4:4 + size]
                raise ValueError("chunked layout not supported")
            if ver in (1, 2):
                rank, cls = b[1], b[2]
                if cls != 1:
                    raise ValueError("only contiguous layouts are supported")
                addr = struct.unpack_from("<Q", b, 8)[0]
                dims = struct.unpack_from("<" + "I" * rank, b, 16)
                size = int(np.prod(dims))
                return self.d[self.base + addr:self.base + addr + size]
        raise ValueError("dataset without a layout message")

    def heap_name(self, heap: int, off: int) -> str:
        if self.d[self.base + heap:self.base + heap + 4] != b"HEAP":
            raise ValueError("bad local heap")
        _, _, seg = self.u("<QQQ", heap + 8)
        p = self.base + seg + off
        return self.d[p:self.d.index(b"\0", p)].decode("ascii")

    def group_entries(self, bt: int, heap: int):
        out = []
        if self.d[self.base + bt:self.base + bt + 4] != b"TREE":
            raise ValueError("bad B-tree node")
        ntype, level, used = self.u("<BBH", bt + 4)
        if ntype != 0:
            raise ValueError("not a group B-tree")
        p = bt + 24 + 8
        for _ in range(used):
            child = self.u("<Q", p)[0]
            p += 16
            if level > 0:
                out += self.group_entries(child, heap)
            else:
                if self.d[self.base + child:self.base + child + 4] != b"SNOD":
                    raise ValueError("bad symbol table node")
                n = self.u("<H", child + 6)[0]
                for e in range(n):
                    name_off, oh = self.u("<QQ", child + 8 + 40 * e)
                    out.append((self.heap_name(heap, name_off), oh))
        return out

    def root(self) -> Node:
        _, oh = struct.unpack_from("<QQ", self.d, self.root_entry)
        return self.obj(oh)


def read(path: str) -> Node:
    """The whole file as a tree of Nodes (group children by name, dataset values as
    numpy arrays or strings, attributes)."""
    with open(path, "rb") as f:
        return _Reader(f.read()).root()
