"""A self-contained HDF5 writer and reader for the multigrid driver's output file.

The reference's `multigrid` binary writes its snapshots with the hdf5 crate
(multigrid/src/system.rs:29-47 creates the root dataset `t`; :86-116 one group per grid with
datasets `x`, `y` of shape (ny, nx), a soft link `t` -> `/t` and the time-extendable datasets
`rho`, `rhou`, `rhov`, `e` of shape (outputs, ny, nx); :591-616 appends one time slice per
output).  No HDF5 library exists in this environment, so this module writes the file format
itself: the same groups, link, dataset names, shapes, element types (f64 little-endian, `t` as
u64) and values, in the format's earliest, most widely readable form:

* superblock version 0 (8-byte offsets and lengths, group leaf K 4, internal K 16);
* groups as symbol tables: object header with a symbol-table message, a version-1 B-tree with
  one leaf node, symbol-table nodes of up to 8 entries sorted by name, and a local heap with the
  names (the soft link's value `/t` too);
* datasets as version-1 object headers holding a dataspace, a datatype, a fill-value message
  (no fill value defined) and a contiguous data-layout message.

What differs from the reference's file: the datasets are contiguous and uncompressed with
maximum shape equal to their shape (the reference's are chunked, deflated and extendable in
time), because the whole run is written at once at the end.  A reader sees the same names,
shapes, types and values.

`read` parses files of exactly this form (and is what the tests use to check the writer).
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
LEAF_K = 4        # symbol-table node capacity is 2 * LEAF_K entries
INTERNAL_K = 16   # group B-tree node capacity is 2 * INTERNAL_K children

# object header message types
MSG_DATASPACE = 0x0001
MSG_DATATYPE = 0x0003
MSG_FILL = 0x0005
MSG_LAYOUT = 0x0008
MSG_SYMBOL_TABLE = 0x0011


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


class SoftLink:
    """A soft link to an absolute path, as a group member."""

    def __init__(self, target: str):
        self.target = target


class _Writer:
    def __init__(self):
        self.buf = bytearray(96)  # superblock, filled in last

    def alloc(self, data: bytes) -> int:
        """Appends `data` at the next 8-byte boundary and returns its address."""
        self.buf += b"\0" * (-len(self.buf) % 8)
        addr = len(self.buf)
        self.buf += data
        return addr

    def patch(self, addr: int, data: bytes) -> None:
        self.buf[addr:addr + len(data)] = data

    # ---- object headers ----
    def object_header(self, messages) -> int:
        body = b""
        for mtype, data in messages:
            data = _pad8(data)
            body += struct.pack("<HHB3x", mtype, len(data), 0) + data
        prefix = struct.pack("<BBHII", 1, 0, len(messages), 1, len(body)) + b"\0" * 4
        return self.alloc(prefix + body)

    # ---- datasets ----
    def dataset(self, arr: np.ndarray) -> int:
        arr = np.ascontiguousarray(arr)
        if arr.dtype == np.float64:
            arr = arr.astype("<f8", copy=False)
            dtype_msg = struct.pack("<B3BI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        elif arr.dtype == np.uint64:
            arr = arr.astype("<u8", copy=False)
            dtype_msg = struct.pack("<B3BI", 0x10, 0, 0, 0, 8) + struct.pack("<HH", 0, 64)
        else:
            raise TypeError(f"unsupported dtype {arr.dtype}")
        rank = arr.ndim
        space = struct.pack("<BBBB4x", 1, rank, 1, 0)
        space += b"".join(struct.pack("<Q", d) for d in arr.shape)
        space += b"".join(struct.pack("<Q", d) for d in arr.shape)  # maximum dimensions
        data_addr = self.alloc(arr.tobytes()) if arr.size else UNDEF
        fill = struct.pack("<BBBB", 2, 2, 2, 0)  # version 2, late allocation, written if set, none defined
        layout = struct.pack("<BBQQ", 3, 1, data_addr, arr.nbytes)
        return self.object_header([(MSG_DATASPACE, space), (MSG_DATATYPE, dtype_msg), (MSG_FILL, fill),
                                   (MSG_LAYOUT, layout)])

    # ---- groups ----
    def group(self, members: dict) -> tuple:
        """Writes a group whose members map names to arrays, dicts (subgroups) or SoftLinks.
        Returns (object header address, B-tree address, local heap address)."""
        names = sorted(members)  # symbol-table nodes are searched by name
        cap = 2 * LEAF_K
        if len(names) > 2 * INTERNAL_K * cap:
            raise ValueError(f"a group holds at most {2 * INTERNAL_K * cap} members in this writer")
        # local heap: offset 0 is the empty string, then the names and link values
        heap = bytearray(b"\0" * 8)

        def put(text: str) -> int:
            off = len(heap)
            heap.extend(_pad8(text.encode() + b"\0"))
            return off

        entries = []
        for name in names:
            m = members[name]
            noff = put(name)
            if isinstance(m, SoftLink):
                entries.append((noff, UNDEF, 2, struct.pack("<I12x", put(m.target))))
            elif isinstance(m, dict):
                oh, bt, hp = self.group(m)
                entries.append((noff, oh, 1, struct.pack("<QQ", bt, hp)))
            else:
                entries.append((noff, self.dataset(np.asarray(m)), 0, b"\0" * 16))
        heap_data = self.alloc(bytes(heap))
        heap_addr = self.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), UNDEF, heap_data))
        # symbol-table nodes of up to 2 LEAF_K entries each, in name order
        nodes = []
        for i in range(0, max(len(entries), 1), cap):
            part = entries[i:i + cap]
            snod = b"SNOD" + struct.pack("<BBH", 1, 0, len(part))
            for noff, oh, cache, scratch in part:
                snod += struct.pack("<QQI4x", noff, oh, cache) + scratch
            snod += b"\0" * (8 + cap * 40 - len(snod))
            nodes.append((self.alloc(snod), part[-1][0] if part else 0))
        # one leaf B-tree node: key 0 is the empty name, child i is symbol-table node i and key
        # i + 1 the heap offset of its greatest name; space for 2K children and 2K + 1 keys
        tree = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(nodes), UNDEF, UNDEF) + struct.pack("<Q", 0)
        for addr, key in nodes:
            tree += struct.pack("<QQ", addr, key)
        tree += b"\0" * (24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8 - len(tree))
        tree_addr = self.alloc(tree)
        oh = self.object_header([(MSG_SYMBOL_TABLE, struct.pack("<QQ", tree_addr, heap_addr))])
        return oh, tree_addr, heap_addr

    def finish(self, root: tuple) -> bytes:
        oh, bt, hp = root
        self.buf += b"\0" * (-len(self.buf) % 8)
        eof = len(self.buf)
        sb = SIGNATURE + struct.pack("<8B", 0, 0, 0, 0, 0, 8, 8, 0)
        sb += struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, oh, 1, bt, hp)  # root group symbol-table entry
        assert len(sb) == 96
        self.patch(0, sb)
        return bytes(self.buf)


def write(path: str, tree: dict) -> None:
    """Writes `tree` (names -> arrays, nested dicts for groups, SoftLink for soft links) as an
    HDF5 file at `path`."""
    w = _Writer()
    root = w.group(tree)
    data = w.finish(root)
    with open(path, "wb") as f:
        f.write(data)


def write_snapshots(path: str, names, grids, times, frames) -> None:
    """The multigrid output file: root dataset `t` (u64, the step number of every output), and per
    grid a group with `x`, `y` (ny, nx), a soft link `t` -> `/t` and `rho`, `rhou`, `rhov`, `e`
    of shape (outputs, ny, nx) (multigrid/src/system.rs:29-47, 86-116, 591-616).  frames[k][b] is
    the (4, ny, nx) state of grid b at output k."""
    tree = {"t": np.asarray(times, dtype=np.uint64)}
    for b, name in enumerate(names):
        g = {"x": np.asarray(grids[b].x, dtype=np.float64), "y": np.asarray(grids[b].y, dtype=np.float64),
             "t": SoftLink("/t")}
        for c, comp in enumerate(("rho", "rhou", "rhov", "e")):
            g[comp] = np.stack([np.asarray(f[b][c], dtype=np.float64) for f in frames])
        tree[name] = g
    write(path, tree)


# ------------------------------------------------------------------------------------------
def read(path: str) -> dict:
    """Reads a file of the form `write` produces into nested dicts of arrays; soft links are
    returned as SoftLink objects.  Checks the signatures and versions it relies on."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != SIGNATURE:
        raise ValueError("not an HDF5 file")
    if buf[8] != 0 or buf[13] != 8 or buf[14] != 8:
        raise ValueError("only superblock version 0 with 8-byte offsets and lengths is read")
    leaf_k, internal_k = struct.unpack_from("<HH", buf, 16)
    eof = struct.unpack_from("<Q", buf, 40)[0]
    if eof != len(buf):
        raise ValueError(f"end-of-file address {eof} differs from the file size {len(buf)}")
    root_oh = struct.unpack_from("<Q", buf, 64)[0]

    def messages(addr):
        version, _, nmsg, _, size = struct.unpack_from("<BBHII", buf, addr)
        if version != 1:
            raise ValueError("only version-1 object headers are read")
        pos, end, out = addr + 16, addr + 16 + size, {}
        for _ in range(nmsg):
            mtype, msize = struct.unpack_from("<HH", buf, pos)
            out[mtype] = buf[pos + 8:pos + 8 + msize]
            pos += 8 + msize
        if pos != end:
            raise ValueError("object header size does not match its messages")
        return out

    def heap_string(heap_data, off):
        end = buf.index(b"\0", heap_data + off)
        return buf[heap_data + off:end].decode()

    def group(tree_addr, heap_addr):
        if buf[heap_addr:heap_addr + 4] != b"HEAP":
            raise ValueError("bad local heap")
        heap_data = struct.unpack_from("<Q", buf, heap_addr + 24)[0]
        if buf[tree_addr:tree_addr + 4] != b"TREE" or buf[tree_addr + 4] != 0 or buf[tree_addr + 5] != 0:
            raise ValueError("only a single leaf group B-tree is read")
        nchild = struct.unpack_from("<H", buf, tree_addr + 6)[0]
        out, prev = {}, None
        for i in range(nchild):
            snod = struct.unpack_from("<Q", buf, tree_addr + 24 + 8 + 16 * i)[0]
            if buf[snod:snod + 4] != b"SNOD":
                raise ValueError("bad symbol-table node")
            n = struct.unpack_from("<H", buf, snod + 6)[0]
            for k in range(n):
                noff, oh, cache = struct.unpack_from("<QQI", buf, snod + 8 + 40 * k)
                name = heap_string(heap_data, noff)
                if prev is not None and not prev < name:
                    raise ValueError("symbol-table entries are not sorted by name")
                prev = name
                if cache == 2:
                    out[name] = SoftLink(heap_string(heap_data, struct.unpack_from("<I", buf, snod + 8 + 40 * k + 24)[0]))
                else:
                    out[name] = obj(oh)
        return out

    def obj(addr):
        msgs = messages(addr)
        if MSG_SYMBOL_TABLE in msgs:
            return group(*struct.unpack_from("<QQ", msgs[MSG_SYMBOL_TABLE], 0))
        space, dtype, layout = msgs[MSG_DATASPACE], msgs[MSG_DATATYPE], msgs[MSG_LAYOUT]
        rank = space[1]
        shape = struct.unpack_from(f"<{rank}Q", space, 8)
        cls, size = dtype[0] & 0x0F, struct.unpack_from("<I", dtype, 4)[0]
        if (cls, size) == (1, 8):
            dt = np.dtype("<f8")
        elif (cls, size) == (0, 8) and not dtype[1] & 0x08:
            dt = np.dtype("<u8")
        else:
            raise ValueError(f"unsupported datatype class {cls} size {size}")
        if layout[0] != 3 or layout[1] != 1:
            raise ValueError("only contiguous layouts are read")
        daddr, nbytes = struct.unpack_from("<QQ", layout, 2)
        count = int(np.prod(shape)) if rank else 1
        if nbytes != count * dt.itemsize:
            raise ValueError("layout size does not match the dataspace")
        if count == 0:
            return np.zeros(shape, dt)
        return np.frombuffer(buf, dt, count, daddr).reshape(shape).copy()

    m = messages(root_oh)
    return group(*struct.unpack_from("<QQ", m[MSG_SYMBOL_TABLE], 0))


def read_flat(path: str) -> dict:
    """`read`, flattened to "group/name" keys with soft links resolved."""
    tree = read(path)
    out = {}

    def walk(node, prefix):
        for name, v in node.items():
            key = prefix + name
            if isinstance(v, dict):
                walk(v, key + "/")
            else:
                out[key] = v
    walk(tree, "")
    for key, v in list(out.items()):
        if isinstance(v, SoftLink):
            out[key] = out[v.target.lstrip("/")]
    return out
