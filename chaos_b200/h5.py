"""A self-contained writer and reader of the HDF5 file format subset the run store needs (no HDF5 library is
installed with this package): the run store's chunk files are HDF5 files (src/Experiments/run_store.jl:1-5, written
there through HDF5.jl, which calls libhdf5).

What is written, following the published HDF5 File Format Specification (version 0 superblock family, the layout
libhdf5 writes by default for files of its earliest format):

* superblock version 0: 8-byte offsets and lengths, group leaf node K = 4, group internal node K = 16;
* object headers version 1 (a 16-byte prefix, 8-byte aligned messages);
* groups in the symbol-table form: a Symbol Table message, a version 1 B-tree of group nodes (as many levels as the
  member count needs), symbol table nodes of up to 2 K entries sorted by name, a local heap holding the names (with
  one free block at its end, whose next-block field holds 1, the end of the free list);
* datasets: Dataspace (version 1), Datatype (version 1), Fill Value (version 2, undefined, late allocation) and
  Data Layout (version 3, contiguous) messages; the raw data little-endian in C order;
* attributes: Attribute messages version 1 in the object header (so one attribute's message stays under 64 KiB).

Element types: int64 / int32 / uint32 / uint8 (fixed-point), float64 / float32 (IEEE), bool (an enum of int8 with
members FALSE = 0 and TRUE = 1, the form libhdf5 users such as h5py and HDF5.jl read as Bool), strings as fixed-length
UTF-8 strings (size max(bytes, 1), null-terminated padding, as HDF5.jl writes a String: size = its byte length), and
string lists as one-dimensional arrays of fixed-length strings.

`write(path, root)` writes a tree of `Group` / `Dataset`; `read(path)` returns the same tree. The reader reads what
the writer writes (and compact layouts); other HDF5 features (version 2 object headers, dense attribute storage,
chunked or filtered datasets, variable-length strings) raise `H5FormatError`.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
LEAF_K = 4
INTERNAL_K = 16
SUPERBLOCK_SIZE = 96
ENTRY_SIZE = 40
OH_PREFIX = 16

MSG_NIL, MSG_DATASPACE, MSG_DATATYPE, MSG_FILL, MSG_LAYOUT, MSG_ATTR, MSG_SYMTAB = 0x0, 0x1, 0x3, 0x5, 0x8, 0xC, 0x11


class H5FormatError(ValueError):
    """A file (or a value) outside the subset of HDF5 this module writes and reads."""


@dataclass
class Dataset:
    """An array stored contiguously; `data` is in file order (C order of the file's extents)."""
    data: np.ndarray
    attrs: dict = field(default_factory=dict)


@dataclass
class Group:
    attrs: dict = field(default_factory=dict)
    members: dict = field(default_factory=dict)

    def require(self, path: str) -> "Group":
        """The group at `path` (slash-separated, relative), created with its parents where missing."""
        g = self
        for part in [p for p in path.split("/") if p]:
            nxt = g.members.get(part)
            if nxt is None:
                nxt = g.members[part] = Group()
            elif not isinstance(nxt, Group):
                raise H5FormatError(f"{part!r} is a dataset, not a group")
            g = nxt
        return g

    def put(self, path: str, obj) -> None:
        """Place a Dataset or Group at `path`, creating the intermediate groups; a taken name raises."""
        head, _, name = path.rstrip("/").rpartition("/")
        g = self.require(head)
        if not name or name in g.members:
            raise H5FormatError(f"name {path!r} is empty or taken")
        g.members[name] = obj


def _pad8(n: int) -> int:
    return (n + 7) & ~7


# ---------------------------------------------------------------- datatypes
def _fixed_type(size: int, signed: bool) -> bytes:
    return struct.pack("<BBBBI", 0x10, 0x08 if signed else 0x00, 0, 0, size) + struct.pack("<HH", 0, 8 * size)


def _float_type(size: int) -> bytes:
    if size == 8:
        sign, eloc, esz, msz, bias = 63, 52, 11, 52, 1023
    else:
        sign, eloc, esz, msz, bias = 31, 23, 8, 23, 127
    head = struct.pack("<BBBBI", 0x11, 0x20, sign, 0, size)
    return head + struct.pack("<HHBBBBI", 0, 8 * size, eloc, esz, 0, msz, bias)


def _string_type(size: int) -> bytes:
    # padding type 0 (null-terminated) in bits 0-3, character set 1 (UTF-8) in bits 4-7
    return struct.pack("<BBBBI", 0x13, 0x10, 0, 0, size)


def _bool_type() -> bytes:
    base = _fixed_type(1, True)
    names = b"FALSE".ljust(8, b"\0") + b"TRUE".ljust(8, b"\0")
    return struct.pack("<BBBBI", 0x18, 2, 0, 0, 1) + base + names + bytes([0, 1])


_NUMERIC = {np.dtype("<i8"): lambda: _fixed_type(8, True), np.dtype("<i4"): lambda: _fixed_type(4, True),
            np.dtype("<u4"): lambda: _fixed_type(4, False), np.dtype("u1"): lambda: _fixed_type(1, False),
            np.dtype("<f8"): lambda: _float_type(8), np.dtype("<f4"): lambda: _float_type(4)}


def _dataspace(dims) -> bytes:
    dims = tuple(int(d) for d in dims)
    return struct.pack("<BBBB4x", 1, len(dims), 0, 0) + b"".join(struct.pack("<Q", d) for d in dims)


def _encode_value(v):
    """(datatype message, dims, raw bytes) of an attribute value or a dataset array."""
    if isinstance(v, (bool, np.bool_)):
        return _bool_type(), (), bytes([1 if v else 0])
    if isinstance(v, str):
        b = v.encode("utf-8")
        if b"\0" in b:
            raise H5FormatError("a string holds a NUL byte")
        size = max(len(b), 1)
        return _string_type(size), (), b.ljust(size, b"\0")
    if isinstance(v, (list, tuple)) and all(isinstance(s, str) for s in v) and (len(v) == 0 or isinstance(v, list)):
        bs = [s.encode("utf-8") for s in v]
        if any(b"\0" in b for b in bs):
            raise H5FormatError("a string holds a NUL byte")
        size = max([len(b) for b in bs] + [1])
        return _string_type(size), (len(bs),), b"".join(b.ljust(size, b"\0") for b in bs)
    if isinstance(v, (int, np.integer)) and not isinstance(v, (np.uint32, np.uint8)):
        return _fixed_type(8, True), (), struct.pack("<q", int(v))
    if isinstance(v, (np.uint32, np.uint8)):
        a = np.asarray(v)
        return _NUMERIC[a.dtype.newbyteorder("<") if a.dtype.itemsize > 1 else a.dtype](), (), a.tobytes()
    if isinstance(v, (float, np.floating)):
        return _float_type(8 if not isinstance(v, np.float32) else 4), (), np.asarray(v).astype(
            "<f8" if not isinstance(v, np.float32) else "<f4").tobytes()
    a = np.asarray(v)
    if a.dtype == np.bool_:
        if a.ndim:
            raise H5FormatError("bool arrays are not written")
        return _encode_value(bool(a))
    dt = a.dtype.newbyteorder("<") if a.dtype.itemsize > 1 else a.dtype
    if dt not in _NUMERIC:
        raise H5FormatError(f"element type {a.dtype} is not written")
    return _NUMERIC[dt](), a.shape, np.ascontiguousarray(a, dtype=dt).tobytes()


def _msg(mtype: int, body: bytes, flags: int = 0) -> bytes:
    n = _pad8(len(body))
    if n > 0xFFFF:
        raise H5FormatError(f"a header message of {n} bytes exceeds 64 KiB")
    return struct.pack("<HHB3x", mtype, n, flags) + body.ljust(n, b"\0")


def _attr_msg(name: str, value) -> bytes:
    nb = name.encode("utf-8") + b"\0"
    dt, dims, raw = _encode_value(value)
    ds = _dataspace(dims)
    body = struct.pack("<BBHHH", 1, 0, len(nb), len(dt), len(ds))
    body += nb.ljust(_pad8(len(nb)), b"\0") + dt.ljust(_pad8(len(dt)), b"\0") + ds.ljust(_pad8(len(ds)), b"\0") + raw
    return _msg(MSG_ATTR, body)


def _object_header(msgs: list[bytes]) -> bytes:
    body = b"".join(msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


# ---------------------------------------------------------------- writing
class _Out:
    """The file image, grown 8 bytes at a time: every structure starts on an 8-byte boundary."""

    def __init__(self):
        self.buf = bytearray(SUPERBLOCK_SIZE)

    def alloc(self, n: int) -> int:
        a = len(self.buf)
        self.buf += bytes(_pad8(n))
        return a

    def put(self, addr: int, b: bytes) -> None:
        self.buf[addr:addr + len(b)] = b


BTREE_NODE_SIZE = 24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8
SNOD_SIZE = 8 + 2 * LEAF_K * ENTRY_SIZE


def _place_dataset(out: _Out, d: Dataset) -> int:
    a = np.asarray(d.data)
    if a.dtype == np.bool_ or a.dtype.kind in "USO":
        raise H5FormatError(f"dataset element type {a.dtype} is not written")
    dt, dims, raw = _encode_value(a)
    attr_msgs = [_attr_msg(k, v) for k, v in d.attrs.items()]
    msgs = [_msg(MSG_DATASPACE, _dataspace(dims)), _msg(MSG_DATATYPE, dt, flags=1),
            _msg(MSG_FILL, struct.pack("<BBBB", 2, 2, 2, 0)), None] + attr_msgs
    hdr = out.alloc(OH_PREFIX + sum(len(m) for m in msgs if m is not None) + 8 + _pad8(18))
    addr = out.alloc(len(raw)) if raw else UNDEF
    if raw:
        out.put(addr, raw)
    msgs[3] = _msg(MSG_LAYOUT, struct.pack("<BBQQ", 3, 1, addr, len(raw)))
    out.put(hdr, _object_header(msgs))
    return hdr


def _place_group(out: _Out, g: Group) -> tuple[int, int, int]:
    """Header, B-tree root and local heap addresses of a group (its members placed after its header)."""
    attr_msgs = [_attr_msg(k, v) for k, v in g.attrs.items()]
    hdr = out.alloc(OH_PREFIX + 8 + 16 + sum(len(m) for m in attr_msgs))
    names = sorted(g.members, key=lambda s: s.encode("utf-8"))
    data = bytearray(8)                       # offset 0: the empty name (the B-trees' left-most key)
    offs = {}
    for nm in names:
        b = nm.encode("utf-8") + b"\0"
        if b"\0" in b[:-1] or b"/" in b[:-1] or nm in (".",):
            raise H5FormatError(f"bad member name {nm!r}")
        offs[nm] = len(data)
        data += b.ljust(_pad8(len(b)), b"\0")
    free = len(data)
    data += struct.pack("<QQ", 1, 16)         # one free block; next-block 1 ends the free list
    heap = out.alloc(32)
    heap_data = out.alloc(len(data))
    out.put(heap, b"HEAP" + struct.pack("<B3xQQQ", 0, len(data), free, heap_data))
    out.put(heap_data, bytes(data))
    entries = []
    for nm in names:
        m = g.members[nm]
        if isinstance(m, Group):
            a, bt, hp = _place_group(out, m)
            entries.append(struct.pack("<QQII", offs[nm], a, 1, 0) + struct.pack("<QQ", bt, hp))
        elif isinstance(m, Dataset):
            entries.append(struct.pack("<QQII16x", offs[nm], _place_dataset(out, m), 0, 0))
        else:
            raise H5FormatError(f"member {nm!r} is neither a Group nor a Dataset")
    nodes = []                                # (address, heap offset of the subtree's last name)
    for i in range(0, len(entries), 2 * LEAF_K):
        chunk = entries[i:i + 2 * LEAF_K]
        a = out.alloc(SNOD_SIZE)
        out.put(a, b"SNOD" + struct.pack("<BxH", 1, len(chunk)) + b"".join(chunk))
        nodes.append((a, offs[names[i + len(chunk) - 1]]))
    level = 0
    while True:
        groups = [nodes[i:i + 2 * INTERNAL_K] for i in range(0, max(len(nodes), 1), 2 * INTERNAL_K)]
        addrs = [out.alloc(BTREE_NODE_SIZE) for _ in groups]
        parents = []
        for j, (a, kids) in enumerate(zip(addrs, groups)):
            left = addrs[j - 1] if j > 0 else UNDEF            # siblings linked: readers may walk a level by them
            right = addrs[j + 1] if j + 1 < len(addrs) else UNDEF
            body = b"TREE" + struct.pack("<BBHQQ", 0, level, len(kids), left, right) + struct.pack("<Q", 0)
            body += b"".join(struct.pack("<QQ", c, k) for c, k in kids)
            out.put(a, body)
            parents.append((a, kids[-1][1] if kids else 0))
        if len(parents) == 1:
            root = parents[0][0]
            break
        nodes, level = parents, level + 1
    out.put(hdr, _object_header([_msg(MSG_SYMTAB, struct.pack("<QQ", root, heap))] + attr_msgs))
    return hdr, root, heap


def image(root: Group) -> bytes:
    """The bytes of an HDF5 file holding `root` as its root group."""
    out = _Out()
    hdr, bt, hp = _place_group(out, root)
    entry = struct.pack("<QQII", 0, hdr, 1, 0) + struct.pack("<QQ", bt, hp)
    sb = SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, len(out.buf), UNDEF) + entry
    assert len(sb) == SUPERBLOCK_SIZE
    out.put(0, sb)
    return bytes(out.buf)


def write(path: str, root: Group) -> None:
    with open(path, "wb") as f:
        f.write(image(root))


# ---------------------------------------------------------------- reading
def _u(fmt: str, buf, off: int):
    if off < 0 or off + struct.calcsize(fmt) > len(buf):
        raise H5FormatError(f"read past the end of the file at {off}")
    return struct.unpack_from(fmt, buf, off)


def _type_len(buf, p: int) -> int:
    """Bytes of the datatype message at p (the classes this module reads)."""
    cls = buf[p] & 0x0F
    if cls == 0:
        return 12
    if cls == 1:
        return 20
    if cls == 3:
        return 8
    raise H5FormatError(f"datatype class {cls} is not read")


def _read_type(buf, p: int):
    cls, ver = buf[p] & 0x0F, buf[p] >> 4
    bf0, bf1 = buf[p + 1], buf[p + 2]
    (size,) = _u("<I", buf, p + 4)
    if ver != 1:
        raise H5FormatError(f"datatype version {ver} is not read")
    if cls == 0:
        if bf0 & 1 or size not in (1, 2, 4, 8):
            raise H5FormatError("big-endian or odd-sized integers are not read")
        return ("num", np.dtype(("<i" if bf0 & 0x08 else "<u") + str(size)))
    if cls == 1:
        if bf0 & 1 or size not in (4, 8):
            raise H5FormatError("big-endian or odd-sized floats are not read")
        return ("num", np.dtype("<f%d" % size))
    if cls == 3:
        return ("str", size)
    if cls == 8:
        nmem = bf0 | (bf1 << 8)
        q = p + 8
        base = _read_type(buf, q)
        q += _type_len(buf, q)
        names = []
        for _ in range(nmem):
            end = buf.index(b"\0", q)
            names.append(bytes(buf[q:end]).decode("ascii"))
            q += _pad8(end - q + 1)
        vals = list(bytes(buf[q:q + nmem * base[1].itemsize]))
        if base[0] == "num" and base[1].itemsize == 1 and size == 1 and dict(zip(names, vals)) == {"FALSE": 0, "TRUE": 1}:
            return ("bool", 1)
        raise H5FormatError(f"enum {names} is not read")
    raise H5FormatError(f"datatype class {cls} is not read")


def _read_space(buf, p: int) -> tuple:
    ver, rank, flags = buf[p], buf[p + 1], buf[p + 2]
    if ver == 1:
        q = p + 8
    elif ver == 2:
        if buf[p + 3] == 2:
            raise H5FormatError("null dataspaces are not read")
        q = p + 4
    else:
        raise H5FormatError(f"dataspace version {ver} is not read")
    return tuple(int(d) for d in _u("<%dQ" % rank, buf, q))


def _decode(buf, q: int, t, dims: tuple):
    count = int(np.prod(dims)) if dims else 1
    if t[0] == "bool":
        if dims:
            raise H5FormatError("bool arrays are not read")
        return bool(buf[q]), 1
    if t[0] == "str":
        size = t[1]
        raw = bytes(buf[q:q + size * count])
        items = [raw[i * size:(i + 1) * size].split(b"\0", 1)[0].decode("utf-8") for i in range(count)]
        if len(dims) > 1:
            raise H5FormatError("string arrays of rank > 1 are not read")
        return (items if dims else items[0]), size * count
    dt = t[1]
    if q + dt.itemsize * count > len(buf):
        raise H5FormatError("data past the end of the file")
    a = np.frombuffer(buf, dt, count, q).reshape(dims).copy()
    if not dims:
        return (a.item() if dt in (np.dtype("<i8"), np.dtype("<f8")) else a[()]), dt.itemsize
    return a, dt.itemsize * count


def _messages(buf, addr: int) -> list:
    ver, _, nmsg, _, size = _u("<BBHII", buf, addr)
    if ver != 1:
        raise H5FormatError(f"object header version {ver} at {addr} is not read")
    p, end, out = addr + OH_PREFIX, addr + OH_PREFIX + size, []
    while p + 8 <= end and len(out) < nmsg:
        mtype, msize = _u("<HH", buf, p)
        if mtype == 0x10:
            raise H5FormatError("continued object headers are not read")
        out.append((mtype, p + 8, msize))
        p += 8 + msize
    return out


def _read_attr(buf, p: int):
    ver, _, nlen, dlen, slen = _u("<BBHHH", buf, p)
    if ver != 1:
        raise H5FormatError(f"attribute message version {ver} is not read")
    q = p + 8
    name = bytes(buf[q:q + nlen - 1]).decode("utf-8")
    q += _pad8(nlen)
    t = _read_type(buf, q)
    q += _pad8(dlen)
    dims = _read_space(buf, q)
    q += _pad8(slen)
    value, nbytes = _decode(buf, q, t, dims)
    return name, value, (q, nbytes)


def _heap_names(buf, heap: int):
    if bytes(buf[heap:heap + 4]) != b"HEAP":
        raise H5FormatError(f"no local heap at {heap}")
    size, _, data = _u("<QQQ", buf, heap + 8)

    def name(off: int) -> str:
        if off >= size:
            raise H5FormatError("name offset past the local heap")
        end = buf.index(b"\0", data + off)
        return bytes(buf[data + off:end]).decode("utf-8")
    return name


def _walk(buf, node: int, out: list, depth: int = 0) -> None:
    if depth > 16 or bytes(buf[node:node + 4]) != b"TREE":
        raise H5FormatError(f"no group B-tree node at {node}")
    ntype, level, used = _u("<BBH", buf, node + 4)
    if ntype != 0:
        raise H5FormatError("not a group B-tree")
    for i in range(used):
        (child,) = _u("<Q", buf, node + 32 + 16 * i)
        if level:
            _walk(buf, child, out, depth + 1)
            continue
        if bytes(buf[child:child + 4]) != b"SNOD":
            raise H5FormatError(f"no symbol table node at {child}")
        (nsym,) = _u("<H", buf, child + 6)
        for j in range(nsym):
            out.append(_u("<QQ", buf, child + 8 + ENTRY_SIZE * j))


def _read_object(buf, addr: int, depth: int = 0):
    if depth > 64:
        raise H5FormatError("groups nested too deep")
    msgs = _messages(buf, addr)
    attrs, where = {}, {}
    for mtype, p, _ in msgs:
        if mtype == MSG_ATTR:
            name, value, loc = _read_attr(buf, p)
            attrs[name], where[name] = value, loc
    kinds = {m[0]: m[1] for m in msgs}
    if MSG_SYMTAB in kinds:
        bt, heap = _u("<QQ", buf, kinds[MSG_SYMTAB])
        name = _heap_names(buf, heap)
        entries = []
        _walk(buf, bt, entries)
        g = Group(attrs=attrs)
        g.attr_locations = where
        for off, hdr in entries:
            g.members[name(off)] = _read_object(buf, hdr, depth + 1)
        return g
    if MSG_LAYOUT in kinds:
        t = _read_type(buf, kinds[MSG_DATATYPE])
        if t[0] != "num":
            raise H5FormatError("only numeric datasets are read")
        dims = _read_space(buf, kinds[MSG_DATASPACE])
        p = kinds[MSG_LAYOUT]
        ver, cls = buf[p], buf[p + 1]
        if ver != 3 or cls not in (0, 1):
            raise H5FormatError(f"data layout version {ver} class {cls} is not read")
        count = int(np.prod(dims)) if dims else 1
        if cls == 1:
            daddr, dsize = _u("<QQ", buf, p + 2)
            if dsize and dsize != count * t[1].itemsize:
                raise H5FormatError("contiguous data size disagrees with the dataspace")
            data = np.zeros(dims, t[1]) if daddr == UNDEF or dsize == 0 else _decode(buf, daddr, t, dims)[0]
        else:
            data = _decode(buf, p + 4, t, dims)[0]
        d = Dataset(data=np.asarray(data), attrs=attrs)
        d.attr_locations = where
        return d
    raise H5FormatError(f"object at {addr} is neither a group nor a dataset")


def read_image(buf) -> Group:
    buf = memoryview(buf).cast("B") if not isinstance(buf, (bytes, bytearray)) else buf
    if bytes(buf[:8]) != SIGNATURE:
        raise H5FormatError("not an HDF5 file (signature)")
    if buf[8] != 0 or buf[13] != 8 or buf[14] != 8:
        raise H5FormatError("only version 0 superblocks with 8-byte offsets and lengths are read")
    (eof,) = _u("<Q", buf, 40)
    if eof > len(buf):
        raise H5FormatError(f"truncated file: end of file address {eof}, {len(buf)} bytes")
    (hdr,) = _u("<Q", buf, 64)
    return _read_object(buf, hdr)


def read(path: str) -> Group:
    with open(path, "rb") as f:
        return read_image(f.read())


def patch_attr(path: str, obj_path: str, name: str, value) -> None:
    """Overwrite, in place, the value of an existing attribute of the object at `obj_path` with a value of the same
    encoded type and size (the run store's `complete` flag)."""
    root = read(path)
    obj = root
    for part in [p for p in obj_path.split("/") if p]:
        obj = obj.members[part]
    if name not in obj.attrs:
        raise H5FormatError(f"no attribute {name!r} at {obj_path!r}")
    old_t, old_dims, old_raw = _encode_value(obj.attrs[name])
    t, dims, raw = _encode_value(value)
    if (t, dims, len(raw)) != (old_t, old_dims, len(old_raw)):
        raise H5FormatError(f"attribute {name!r}: the new value has another type or size")
    q, nbytes = obj.attr_locations[name]
    with open(path, "r+b") as f:
        f.seek(q)
        f.write(raw)
