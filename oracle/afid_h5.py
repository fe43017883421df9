"""Oracle for the checkpoint container: a pure-Python restatement of the subset of the HDF5 file
format that the reference's continua files use.

This module is test infrastructure, never the product: the tests use it to read the files that the
library's native writer produces and to write files that the native reader must accept.

The reference writes its restart files through the HDF5 library with default property lists:
one dataset 'var' of H5T_NATIVE_DOUBLE per field with Fortran dims (nx, nym, nzm), contiguous
storage (the chunked variant is commented out, h5tools/HdfRoutines.F90:428-490, refined grid
:530-600), and continua_master.h5 with one-element datasets (HdfSerialWriteIntScalar /
HdfSerialWriteRealScalar, h5tools/HdfRoutines.F90:25-96; names WriteFlowField.F90:54-81).
Default property lists give a version-0 superblock, version-1 object headers and a symbol-table
root group.  The layouts below follow the published HDF5 File Format Specification (version 3.0,
The HDF Group): superblock (II.A), symbol table entry (III.C), version-1 B-tree (III.A.1), symbol
table node (III.B), local heap (III.D), object headers version 1 and 2 (IV.A.1), and the
dataspace (IV.A.2.b), datatype (IV.A.2.d), fill value (IV.A.2.f), link (IV.A.2.g), data layout
(IV.A.2.i), continuation (IV.A.2.q) and symbol table (IV.A.2.r) messages.

Reader scope: superblock versions 0-3, object header versions 1 and 2 with continuation chunks,
symbol-table groups and compact link-message groups, simple and scalar dataspaces, fixed-point and
IEEE floating-point datatypes of either byte order, contiguous and compact layouts.  Chunked
storage, filters and dense link storage raise NotImplementedError.

Parity pin: the reader is checked against a file written by the HDF5 library itself (the MATLAB
7.3 test file that ships with scipy, when present) and against the native writer's files.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


@dataclass
class Dataset:
    name: str
    shape: tuple
    dtype: np.dtype
    address: int = UNDEF          # contiguous data address (UNDEF: not allocated)
    size: int = 0
    compact: bytes | None = None
    attributes: dict = field(default_factory=dict)


class H5File:
    """Read-only view of an HDF5 file held in memory."""

    def __init__(self, path: str):
        with open(path, "rb") as f:
            self.buf = f.read()
        self.base = self._find_superblock()
        self._parse_superblock()

    # --- primitive reads -------------------------------------------------------------------
    def _u(self, pos: int, n: int) -> int:
        return int.from_bytes(self.buf[pos:pos + n], "little")

    def _addr(self, pos: int) -> int:
        return self._u(pos, self.so)

    def _len(self, pos: int) -> int:
        return self._u(pos, self.sl)

    def _find_superblock(self) -> int:
        # the superblock sits at 0, 512, 1024, 2048, ... (user block before it)
        pos = 0
        while pos + 8 <= len(self.buf):
            if self.buf[pos:pos + 8] == SIGNATURE:
                return pos
            pos = 512 if pos == 0 else pos * 2
        raise ValueError("not an HDF5 file")

    def _parse_superblock(self):
        p = self.base + 8
        self.sb_version = self.buf[p]
        if self.sb_version in (0, 1):
            self.so, self.sl = self.buf[p + 5], self.buf[p + 6]
            q = p + 8 + 4 + 4           # leaf K, internal K, consistency flags
            if self.sb_version == 1:
                q += 4                  # indexed storage K + reserved
            base_addr = self._u(q, self.so)
            q += 4 * self.so            # base, free-space, end-of-file, driver block addresses
            # root group symbol table entry
            self.root_header = self._u(q + self.so, self.so)
            cache = self._u(q + 2 * self.so, 4)
            self.root_scratch = None
            if cache == 1:
                sp = q + 2 * self.so + 8
                self.root_scratch = (self._u(sp, self.so), self._u(sp + self.so, self.so))
            self.addr_base = base_addr
        elif self.sb_version in (2, 3):
            self.so, self.sl = self.buf[p + 1], self.buf[p + 2]
            q = p + 4
            self.addr_base = self._u(q, self.so)
            self.root_header = self._u(q + 3 * self.so, self.so)
            self.root_scratch = None
        else:
            raise NotImplementedError(f"superblock version {self.sb_version}")

    def _abs(self, addr: int) -> int:
        return self.addr_base + addr

    # --- object headers --------------------------------------------------------------------
    def messages(self, addr: int):
        """(type, flags, body bytes) of every message of the object header at addr."""
        out = []
        p = self._abs(addr)
        if self.buf[p:p + 4] == b"OHDR":
            flags = self.buf[p + 5]
            q = p + 6
            if flags & 0x20:
                q += 16                 # access/modification/change/birth times
            if flags & 0x10:
                q += 4                  # attribute phase change values
            width = 1 << (flags & 3)
            size0 = self._u(q, width)
            q += width
            chunks = [(q, size0, True)]
            order = bool(flags & 0x04)
            while chunks:
                start, size, first = chunks.pop(0)
                r, end = start, start + size
                if not first:
                    assert self.buf[r:r + 4] == b"OCHK", "bad continuation chunk"
                    r += 4
                    end -= 4            # checksum
                while r + 4 <= end:
                    mtype, msize, mflags = self.buf[r], self._u(r + 1, 2), self.buf[r + 3]
                    r += 4 + (2 if order else 0)
                    body = self.buf[r:r + msize]
                    r += msize
                    if mtype == 0x10:
                        chunks.append((self._abs(self._addr(r - msize)), self._len(r - msize + self.so), False))
                    else:
                        out.append((mtype, mflags, body))
        else:
            version = self.buf[p]
            if version != 1:
                raise NotImplementedError(f"object header version {version}")
            nmsg = self._u(p + 2, 2)
            size0 = self._u(p + 8, 4)
            chunks = [(p + 16, size0)]
            while chunks and len(out) < nmsg:
                start, size = chunks.pop(0)
                r, end = start, start + size
                while r + 8 <= end:
                    mtype, msize, mflags = self._u(r, 2), self._u(r + 2, 2), self.buf[r + 4]
                    body = self.buf[r + 8:r + 8 + msize]
                    r += 8 + msize
                    if mtype == 0x10:
                        chunks.append((self._abs(int.from_bytes(body[:self.so], "little")),
                                       int.from_bytes(body[self.so:self.so + self.sl], "little")))
                    else:
                        out.append((mtype, mflags, body))
        return out

    # --- groups ----------------------------------------------------------------------------
    def _heap_data(self, heap_addr: int) -> int:
        p = self._abs(heap_addr)
        assert self.buf[p:p + 4] == b"HEAP", "bad local heap"
        return self._abs(self._addr(p + 8 + 2 * self.sl))

    def _cstr(self, pos: int) -> str:
        end = self.buf.index(b"\0", pos)
        return self.buf[pos:end].decode()

    def _btree_group(self, btree_addr: int, heap_data: int, out: dict):
        p = self._abs(btree_addr)
        assert self.buf[p:p + 4] == b"TREE", "bad B-tree node"
        ntype, level, used = self.buf[p + 4], self.buf[p + 5], self._u(p + 6, 2)
        assert ntype == 0, "not a group B-tree"
        q = p + 8 + 2 * self.so + self.sl            # siblings, then key 0
        for _ in range(used):
            child = self._addr(q)
            q += self.so + self.sl
            if level > 0:
                self._btree_group(child, heap_data, out)
            else:
                self._snod(child, heap_data, out)

    def _snod(self, addr: int, heap_data: int, out: dict):
        p = self._abs(addr)
        assert self.buf[p:p + 4] == b"SNOD", "bad symbol table node"
        n = self._u(p + 6, 2)
        q = p + 8
        esize = 2 * self.so + 24
        for i in range(n):
            e = q + i * esize
            name = self._cstr(heap_data + self._u(e, self.so))
            out[name] = self._u(e + self.so, self.so)

    def links(self, header_addr: int) -> dict:
        """name -> object header address for the group whose header is at header_addr."""
        out: dict = {}
        for mtype, _, body in self.messages(header_addr):
            if mtype == 0x11:                         # symbol table
                btree = int.from_bytes(body[:self.so], "little")
                heap = int.from_bytes(body[self.so:2 * self.so], "little")
                self._btree_group(btree, self._heap_data(heap), out)
            elif mtype == 0x06:                       # link (compact storage)
                flags = body[1]
                r = 2
                if flags & 0x08:
                    ltype = body[r]
                    r += 1
                else:
                    ltype = 0
                if flags & 0x04:
                    r += 8
                if flags & 0x10:
                    r += 1
                nlen_w = 1 << (flags & 3)
                nlen = int.from_bytes(body[r:r + nlen_w], "little")
                r += nlen_w
                name = body[r:r + nlen].decode()
                r += nlen
                if ltype == 0:
                    out[name] = int.from_bytes(body[r:r + self.so], "little")
            elif mtype == 0x02:                       # link info
                flags = body[1]
                r = 2 + (8 if flags & 1 else 0)
                fheap = int.from_bytes(body[r:r + self.so], "little")
                if fheap != UNDEF and fheap != (1 << (8 * self.so)) - 1:
                    raise NotImplementedError("dense link storage")
        return out

    def root(self) -> dict:
        return self.links(self.root_header)

    def resolve(self, path: str) -> int:
        """Object header address of a '/'-separated path below the root group."""
        addr = self.root_header
        for comp in path.split("/"):
            addr = self.links(addr)[comp]
        return addr

    def is_group(self, path: str) -> bool:
        return any(t in (0x11, 0x02, 0x06) for t, _, _ in self.messages(self.resolve(path)))

    # --- datasets --------------------------------------------------------------------------
    def dataset(self, name: str) -> Dataset:
        addr = self.resolve(name)
        shape, dtype, ds = None, None, Dataset(name, (), np.dtype("f8"))
        for mtype, _, b in self.messages(addr):
            if mtype == 0x01:
                shape = self._dataspace(b)
            elif mtype == 0x03:
                dtype = self._datatype(b)
            elif mtype == 0x08:
                self._layout(b, ds)
            elif mtype == 0x0B:
                raise NotImplementedError("filter pipeline")
        ds.shape, ds.dtype = shape, dtype
        return ds

    def _dataspace(self, b: bytes) -> tuple:
        version, rank, flags = b[0], b[1], b[2]
        if version == 1:
            r = 8
        elif version == 2:
            if b[3] == 0:
                return ()
            if b[3] == 2:
                return (0,)
            r = 4
        else:
            raise NotImplementedError(f"dataspace version {version}")
        return tuple(int.from_bytes(b[r + i * self.sl:r + (i + 1) * self.sl], "little") for i in range(rank))

    @staticmethod
    def _datatype(b: bytes) -> np.dtype:
        cls = b[0] & 0x0F
        bits0 = b[1]
        size = int.from_bytes(b[4:8], "little")
        order = ">" if bits0 & 1 else "<"
        if cls == 0:
            signed = bool(bits0 & 0x08)
            return np.dtype(f"{order}{'i' if signed else 'u'}{size}")
        if cls == 1:
            return np.dtype(f"{order}f{size}")
        raise NotImplementedError(f"datatype class {cls}")

    def _layout(self, b: bytes, ds: Dataset):
        version = b[0]
        if version in (1, 2):
            rank, cls = b[1], b[2]
            r = 8
            if cls == 2:
                raise NotImplementedError("chunked storage")
            if cls == 1:
                ds.address = int.from_bytes(b[r:r + self.so], "little")
                ds.size = -1
            else:
                r += self.so if cls == 1 else 0
                r += 4 * rank
                n = int.from_bytes(b[r:r + 4], "little")
                ds.compact = b[r + 4:r + 4 + n]
        elif version in (3, 4):
            cls = b[1]
            if cls == 0:
                n = int.from_bytes(b[2:4], "little")
                ds.compact = b[4:4 + n]
            elif cls == 1:
                ds.address = int.from_bytes(b[2:2 + self.so], "little")
                ds.size = int.from_bytes(b[2 + self.so:2 + self.so + self.sl], "little")
            else:
                raise NotImplementedError("chunked or virtual storage")
        else:
            raise NotImplementedError(f"layout version {version}")

    def read(self, name: str) -> np.ndarray:
        ds = self.dataset(name)
        count = int(np.prod(ds.shape)) if ds.shape else 1
        nbytes = count * ds.dtype.itemsize
        if ds.compact is not None:
            raw = ds.compact[:nbytes]
        elif ds.address == UNDEF:
            raw = bytes(nbytes)      # never written: the default fill value is zero
        else:
            p = self._abs(ds.address)
            raw = self.buf[p:p + nbytes]
        return np.frombuffer(raw, dtype=ds.dtype, count=count).reshape(ds.shape).astype(ds.dtype.newbyteorder("="))


def read(path: str, name: str) -> np.ndarray:
    return H5File(path).read(name)


def names(path: str) -> list:
    return sorted(H5File(path).root())


# --- writer of the newer layout (superblock version 2, version-2 object headers, link messages) ---
# Used by the tests to hand the native reader a file of the layout that the HDF5 library writes
# with the latest-format setting; the version-0 layout is what the native writer produces.

def lookup3(data: bytes, initval: int = 0) -> int:
    """Bob Jenkins' lookup3 hashlittle (public domain, 2006), the checksum of HDF5 metadata."""
    m = 0xFFFFFFFF

    def rot(x, k):
        return ((x << k) | (x >> (32 - k))) & m

    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & m
    i = 0
    while n > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & m
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & m
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & m
        a = (a - c) & m; a ^= rot(c, 4); c = (c + b) & m
        b = (b - a) & m; b ^= rot(a, 6); a = (a + c) & m
        c = (c - b) & m; c ^= rot(b, 8); b = (b + a) & m
        a = (a - c) & m; a ^= rot(c, 16); c = (c + b) & m
        b = (b - a) & m; b ^= rot(a, 19); a = (a + c) & m
        c = (c - b) & m; c ^= rot(b, 4); b = (b + a) & m
        n -= 12
        i += 12
    if n == 0:
        return c
    tail = data[i:i + n] + bytes(12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & m
    b = (b + int.from_bytes(tail[4:8], "little")) & m
    c = (c + int.from_bytes(tail[8:12], "little")) & m
    c ^= b; c = (c - rot(b, 14)) & m
    a ^= c; a = (a - rot(c, 11)) & m
    b ^= a; b = (b - rot(a, 25)) & m
    c ^= b; c = (c - rot(b, 16)) & m
    a ^= c; a = (a - rot(c, 4)) & m
    b ^= a; b = (b - rot(a, 14)) & m
    c ^= b; c = (c - rot(b, 24)) & m
    return c


def _datatype_msg(dt: np.dtype) -> bytes:
    order = 1 if dt.byteorder == ">" else 0
    if dt.kind == "f":
        if dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            sign = 63
        else:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            sign = 31
        return bytes([0x11, 0x20 | order, sign, 0]) + struct.pack("<I", dt.itemsize) + props
    signed = 0x08 if dt.kind == "i" else 0
    return bytes([0x10, order | signed, 0, 0]) + struct.pack("<I", dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)


def _ohdr_v2(msgs) -> bytes:
    body = b"".join(bytes([t]) + struct.pack("<H", len(m)) + b"\0" + m for t, m in msgs)
    head = b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body))   # chunk-0 size in 4 bytes
    blob = head + body
    return blob + struct.pack("<I", lookup3(blob))


def write_v2(path: str, datasets: dict, compact: tuple = ()) -> None:
    """Superblock version 2, root group of link messages, one version-2 object header per dataset;
    datasets named in compact use compact storage, the others contiguous storage."""
    so = 8
    items = [(k, np.ascontiguousarray(v)) for k, v in datasets.items()]
    sb_len = 48
    # sizes of dataset headers do not depend on addresses of raw data of fixed length
    def ds_msgs(a, addr):
        space = bytes([2, a.ndim, 0, 1]) + b"".join(struct.pack("<Q", d) for d in a.shape)
        fill = bytes([3, 0x0A])
        if addr is None:
            raw = a.tobytes()
            layout = bytes([3, 0]) + struct.pack("<H", len(raw)) + raw
        else:
            layout = bytes([3, 1]) + struct.pack("<QQ", addr, a.nbytes)
        return [(0x01, space), (0x03, _datatype_msg(a.dtype)), (0x05, fill), (0x08, layout)]

    ds_headers_len = [len(_ohdr_v2(ds_msgs(a, None if k in compact else 0))) for k, a in items]
    link_msgs = [(0x02, bytes([0, 0]) + struct.pack("<QQ", UNDEF, UNDEF)), (0x0A, bytes([0, 0]))]
    root_probe = _ohdr_v2(link_msgs + [(0x06, bytes([1, 0x00, len(k.encode())]) + k.encode() + bytes(so))
                                       for k, _ in items])
    a_root = sb_len
    pos = a_root + len(root_probe)
    a_ds = []
    for n in ds_headers_len:
        a_ds.append(pos)
        pos += n
    raw_addr = {}
    for k, a in items:
        if k not in compact:
            raw_addr[k] = pos
            pos += a.nbytes
    eof = pos
    root = _ohdr_v2(link_msgs + [(0x06, bytes([1, 0x00, len(k.encode())]) + k.encode() + struct.pack("<Q", a_ds[i]))
                                 for i, (k, _) in enumerate(items)])
    sb = SIGNATURE + bytes([2, so, 8, 0]) + struct.pack("<QQQQ", 0, UNDEF, eof, a_root)
    sb += struct.pack("<I", lookup3(sb))
    out = bytearray(sb + root)
    for k, a in items:
        out += _ohdr_v2(ds_msgs(a, None if k in compact else raw_addr[k]))
    for k, a in items:
        if k not in compact:
            out += a.tobytes()
    assert len(out) == eof
    with open(path, "wb") as f:
        f.write(out)


# --- writer of the version-0 layout (what the HDF5 library writes with default properties) ------
# An independent restatement of the layout the library's native writer produces, byte for byte:
# superblock v0 with the root symbol table entry (cache type 1), root object header v1 with a
# symbol table message, a local heap ("" at 0, names padded to 8 bytes, empty free list = 1), one
# group B-tree leaf node allocated at 2K = 32 children, symbol table nodes of 2K = 8 entries sorted
# by name, dataset object headers v1 (dataspace v1, datatype v1, fill value v2, layout v3
# contiguous), then the raw data of each dataset in header order, each padded to 8 bytes.

def _pad8(n: int) -> int:
    return (n + 7) & ~7


def _ohdr_v1(msgs) -> bytes:
    body = b""
    for t, m in msgs:
        flags = 1 if t in (0x03, 0x11) else 0
        body += struct.pack("<HHB3x", t, _pad8(len(m)), flags) + m + bytes(_pad8(len(m)) - len(m))
    return struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + bytes(4) + body


def _dataset_msgs(a: np.ndarray, raw_addr: int) -> list:
    space = bytes([1, a.ndim, 0, 0, 0, 0, 0, 0]) + b"".join(struct.pack("<Q", d) for d in a.shape)
    fill = bytes([2, 2, 2, 1, 0, 0, 0, 0])
    layout = bytes([3, 1]) + struct.pack("<QQ", raw_addr, a.nbytes)
    return [(0x01, space), (0x03, _datatype_msg(a.dtype)), (0x05, fill), (0x08, layout)]


def write_v0_tree(path: str, datasets: dict) -> None:
    """write_v0 with nested groups: '/' in a name nests, a None value is an (empty) group.  Per
    group, in depth-first order from the root: object header, local heap, B-tree nodes (root
    level first; a level-l node has up to 32 level l-1 children), symbol table nodes; then every
    dataset header and every dataset's raw data in the order given."""
    K_LEAF, K_INT = 4, 16
    items = list(datasets.items())

    def new_group():
        return {"members": {}, "groups": {}}

    root = new_group()
    for i, (name, a) in enumerate(items):      # the groups, in order of first appearance
        g = root
        for comp in name.split("/")[:-1]:
            g = g["groups"].setdefault(comp, new_group())

    def register(g):                             # a group is a member of its parent
        for comp, child in g["groups"].items():
            g["members"][comp] = ("g", child)
            register(child)
    for i, (name, a) in enumerate(items):
        parts = name.split("/")
        g = root
        for comp in parts[:-1]:
            g = g["groups"][comp]
        if a is None:
            g["groups"].setdefault(parts[-1], new_group())
        else:
            g["members"][parts[-1]] = ("d", i)
    register(root)

    snod_size = 8 + 2 * K_LEAF * 40
    btree_size = 24 + (2 * K_INT + 1) * 8 + 2 * K_INT * 8
    order = []          # groups in placement order

    def place(g, pos):
        g["names"] = sorted(g["members"], key=lambda k: k.encode())
        heap = bytearray(8)
        g["off"] = {}
        for nm in g["names"]:
            g["off"][nm] = len(heap)
            b = nm.encode()
            heap += b + bytes(_pad8(len(b) + 1) - len(b))
        g["heap"] = heap
        nsnod = (len(g["names"]) + 2 * K_LEAF - 1) // (2 * K_LEAF)
        counts = [max(1, (nsnod + 2 * K_INT - 1) // (2 * K_INT))]
        while counts[-1] > 1:
            counts.append((counts[-1] + 2 * K_INT - 1) // (2 * K_INT))
        g["a_oh"] = pos
        pos += 40
        g["a_heap"] = pos
        pos += 32 + len(heap)
        g["levels"] = [[] for _ in counts]
        for lev in range(len(counts) - 1, -1, -1):
            for _ in range(counts[lev]):
                g["levels"][lev].append(pos)
                pos += btree_size
        g["a_snod"] = pos
        g["nsnod"] = nsnod
        pos += nsnod * snod_size
        order.append(g)
        for comp in g["groups"]:
            pos = place(g["groups"][comp], pos)
        return pos

    pos = place(root, 96)
    a_ds = {}
    for i, (k, a) in enumerate(items):
        if a is None:
            continue
        a_ds[i] = pos
        pos += len(_ohdr_v1(_dataset_msgs(np.ascontiguousarray(a), 0)))
    a_raw = {}
    for i, (k, a) in enumerate(items):
        if a is None:
            continue
        a_raw[i] = pos
        pos += _pad8(np.ascontiguousarray(a).nbytes)
    eof = pos
    out = bytearray(SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", K_LEAF, K_INT, 0))
    out += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    out += struct.pack("<QQII", 0, root["a_oh"], 1, 0) + struct.pack("<QQ", root["levels"][-1][0], root["a_heap"])
    for g in order:
        assert len(out) == g["a_oh"]
        out += _ohdr_v1([(0x11, struct.pack("<QQ", g["levels"][-1][0], g["a_heap"]))])
        out += b"HEAP" + bytes(4) + struct.pack("<QQQ", len(g["heap"]), 1, g["a_heap"] + 32) + g["heap"]
        names = g["names"]
        n = len(names)
        child_addr = [g["a_snod"] + c * snod_size for c in range(g["nsnod"])]
        child_key = [g["off"][names[min(n, (c + 1) * 2 * K_LEAF) - 1]] for c in range(g["nsnod"])]
        nodes_bytes = {}
        for lev, nodes in enumerate(g["levels"]):
            nxt_addr, nxt_key = [], []
            for k_, b in enumerate(nodes):
                lo, hi = k_ * 2 * K_INT, min(len(child_addr), (k_ + 1) * 2 * K_INT)
                left = nodes[k_ - 1] if k_ > 0 else UNDEF
                right = nodes[k_ + 1] if k_ + 1 < len(nodes) else UNDEF
                bt = bytearray(b"TREE" + bytes([0, lev]) + struct.pack("<HQQ", hi - lo, left, right))
                bt += struct.pack("<Q", 0)
                for c in range(lo, hi):
                    bt += struct.pack("<QQ", child_addr[c], child_key[c])
                nodes_bytes[b] = bytes(bt) + bytes(btree_size - len(bt))
                nxt_addr.append(b)
                nxt_key.append(child_key[hi - 1] if hi > lo else 0)
            child_addr, child_key = nxt_addr, nxt_key
        for b in sorted(nodes_bytes):
            out += nodes_bytes[b]
        for c in range(g["nsnod"]):
            lo, hi = c * 2 * K_LEAF, min(n, (c + 1) * 2 * K_LEAF)
            sn = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", hi - lo))
            for nm in names[lo:hi]:
                kind, ref = g["members"][nm]
                addr = a_ds[ref] if kind == "d" else ref["a_oh"]
                sn += struct.pack("<QQII", g["off"][nm], addr, 0, 0) + bytes(16)
            out += sn + bytes(snod_size - len(sn))
    for i, (k, a) in enumerate(items):
        if a is not None:
            out += _ohdr_v1(_dataset_msgs(np.ascontiguousarray(a), a_raw[i]))
    for i, (k, a) in enumerate(items):
        if a is not None:
            b = np.ascontiguousarray(a)
            out += b.tobytes() + bytes(_pad8(b.nbytes) - b.nbytes)
    assert len(out) == eof, (len(out), eof)
    with open(path, "wb") as f:
        f.write(out)


def write_v0(path: str, datasets: dict) -> None:
    """float64 / int32 datasets (little-endian), names sorted as C strcmp orders them."""
    K_LEAF, K_INT = 4, 16
    items = [(k, np.ascontiguousarray(v)) for k, v in datasets.items()]
    for k, a in items:
        assert a.dtype in (np.dtype("<f8"), np.dtype("<i4")), (k, a.dtype)
    order = sorted(range(len(items)), key=lambda i: items[i][0].encode())
    heap = bytearray(8)
    name_off = {}
    for i in order:
        name_off[i] = len(heap)
        nm = items[i][0].encode()
        heap += nm + bytes(_pad8(len(nm) + 1) - len(nm))
    nsnod = (len(items) + 2 * K_LEAF - 1) // (2 * K_LEAF)
    snod_size = 8 + 2 * K_LEAF * 40
    btree_size = 24 + (2 * K_INT + 1) * 8 + 2 * K_INT * 8
    a_root = 96
    a_heap = a_root + 40
    a_heapdata = a_heap + 32
    a_btree = a_heapdata + len(heap)
    a_snod = a_btree + btree_size
    pos = a_snod + nsnod * snod_size
    a_oh = []
    for k, a in items:
        a_oh.append(pos)
        pos += len(_ohdr_v1(_dataset_msgs(a, 0)))
    a_raw = []
    for k, a in items:
        a_raw.append(pos)
        pos += _pad8(a.nbytes)
    eof = pos
    out = bytearray(SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", K_LEAF, K_INT, 0))
    out += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    out += struct.pack("<QQII", 0, a_root, 1, 0) + struct.pack("<QQ", a_btree, a_heap)
    assert len(out) == a_root
    out += _ohdr_v1([(0x11, struct.pack("<QQ", a_btree, a_heap))])
    out += b"HEAP" + bytes(4) + struct.pack("<QQQ", len(heap), 1, a_heapdata) + heap
    bt = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", nsnod, UNDEF, UNDEF) + struct.pack("<Q", 0))
    for c in range(nsnod):
        last = order[min(len(items), (c + 1) * 2 * K_LEAF) - 1]
        bt += struct.pack("<QQ", a_snod + c * snod_size, name_off[last])
    out += bt + bytes(btree_size - len(bt))
    for c in range(nsnod):
        sn = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", min(len(items), (c + 1) * 2 * K_LEAF) - c * 2 * K_LEAF))
        for i in order[c * 2 * K_LEAF:(c + 1) * 2 * K_LEAF]:
            sn += struct.pack("<QQII", name_off[i], a_oh[i], 0, 0) + bytes(16)
        out += sn + bytes(snod_size - len(sn))
    for (k, a), r in zip(items, a_raw):
        out += _ohdr_v1(_dataset_msgs(a, r))
    for k, a in items:
        out += a.tobytes() + bytes(_pad8(a.nbytes) - a.nbytes)
    assert len(out) == eof
    with open(path, "wb") as f:
        f.write(out)
