"""The HDF5 writer of the driver's output file (summationbyparts_b200/hdf5.py) on the CPU: round
trips through the module's own reader, the byte layout of the structures it relies on, checked
field by field against the format (superblock version 0, version-1 object headers and B-trees,
symbol-table nodes, local heaps), and the reference's file structure (multigrid/src/system.rs:29-47,
86-116, 591-616)."""
import struct
import types

import numpy as np
import pytest

from summationbyparts_b200 import hdf5


def _tree(rng, ngroups):
    tree = {"t": np.arange(5, dtype=np.uint64) * 7}
    for g in range(ngroups):
        tree[f"block{g:02d}"] = {"x": rng.random((3, 4)), "y": rng.random((3, 4)), "t": hdf5.SoftLink("/t"),
                                 "rho": rng.random((5, 3, 4)), "empty": np.zeros((0, 3))}
    return tree


@pytest.mark.parametrize("ngroups", [0, 1, 7, 8, 9, 40])
def test_round_trip(tmp_path, ngroups):
    rng = np.random.default_rng(ngroups)
    tree = _tree(rng, ngroups)
    path = str(tmp_path / "f.hdf")
    hdf5.write(path, tree)
    back = hdf5.read(path)
    assert sorted(back) == sorted(tree)
    np.testing.assert_array_equal(back["t"], tree["t"])
    assert back["t"].dtype == np.dtype("<u8")
    for g in range(ngroups):
        name = f"block{g:02d}"
        assert sorted(back[name]) == sorted(tree[name])
        assert isinstance(back[name]["t"], hdf5.SoftLink) and back[name]["t"].target == "/t"
        for k in ("x", "y", "rho", "empty"):
            assert back[name][k].dtype == np.dtype("<f8") and back[name][k].shape == tree[name][k].shape
            np.testing.assert_array_equal(back[name][k], tree[name][k])
    flat = hdf5.read_flat(path)
    for g in range(ngroups):
        np.testing.assert_array_equal(flat[f"block{g:02d}/t"], tree["t"])


def test_byte_layout(tmp_path):
    path = str(tmp_path / "f.hdf")
    hdf5.write(path, {"b": {"v": np.array([[1.5, -2.0]]), "t": hdf5.SoftLink("/t")}, "t": np.array([3], np.uint64)})
    buf = open(path, "rb").read()
    # superblock version 0
    assert buf[:8] == b"\x89HDF\r\n\x1a\n"
    assert tuple(buf[8:16]) == (0, 0, 0, 0, 0, 8, 8, 0)
    assert struct.unpack_from("<HHI", buf, 16) == (4, 16, 0)
    base, freesp, eof, driver = struct.unpack_from("<QQQQ", buf, 24)
    assert (base, freesp, eof, driver) == (0, hdf5.UNDEF, len(buf), hdf5.UNDEF)
    name_off, oh, cache = struct.unpack_from("<QQI", buf, 56)
    btree, heap = struct.unpack_from("<QQ", buf, 80)
    assert name_off == 0 and cache == 1
    # root object header: version 1, one symbol-table message naming the same B-tree and heap
    version, _, nmsg, refcount, size = struct.unpack_from("<BBHII", buf, oh)
    assert (version, nmsg, refcount, size) == (1, 1, 1, 24)
    assert struct.unpack_from("<HHB", buf, oh + 16) == (0x0011, 16, 0)
    assert struct.unpack_from("<QQ", buf, oh + 24) == (btree, heap)
    # every structure starts 8-byte aligned
    for addr in (oh, btree, heap):
        assert addr % 8 == 0
    # local heap: offset 0 holds the empty string; names are null-terminated, 8-byte padded
    assert buf[heap:heap + 5] == b"HEAP\0"
    seg_size, free, seg = struct.unpack_from("<QQQ", buf, heap + 8)
    assert free == hdf5.UNDEF and buf[seg] == 0 and seg_size % 8 == 0
    # B-tree: group node type 0, leaf, one child; key 0 = "", key 1 = the last name ("t")
    assert buf[btree:btree + 4] == b"TREE" and struct.unpack_from("<BBH", buf, btree + 4) == (0, 0, 1)
    k0, child, k1 = struct.unpack_from("<QQQ", buf, btree + 24)
    assert k0 == 0 and buf[seg + k1:seg + k1 + 2] == b"t\0"
    # symbol-table node: version 1, two entries in name order ("b" < "t")
    assert buf[child:child + 4] == b"SNOD" and struct.unpack_from("<BBH", buf, child + 4) == (1, 0, 2)
    names = []
    for k in range(2):
        noff, _, _ = struct.unpack_from("<QQI", buf, child + 8 + 40 * k)
        names.append(buf[seg + noff:buf.index(b"\0", seg + noff)].decode())
    assert names == ["b", "t"]


def test_dataset_messages():
    w = hdf5._Writer()
    addr = w.dataset(np.array([[1.0, 2.0, 3.0]]))
    msgs = {}
    version, _, nmsg, _, size = struct.unpack_from("<BBHII", w.buf, addr)
    pos = addr + 16
    for _ in range(nmsg):
        t, n = struct.unpack_from("<HH", w.buf, pos)
        msgs[t] = bytes(w.buf[pos + 8:pos + 8 + n])
        pos += 8 + n
    assert version == 1 and pos == addr + 16 + size
    # dataspace v1: rank 2, maximum dimensions present and equal
    assert msgs[1][:4] == bytes([1, 2, 1, 0]) and struct.unpack_from("<4Q", msgs[1], 8) == (1, 3, 1, 3)
    # IEEE f64 little-endian: class 1 version 1, implied-MSB mantissa, sign at bit 63, exponent
    # 52..62 with bias 1023, mantissa 0..51
    assert msgs[3][:8] == bytes([0x11, 0x20, 63, 0, 8, 0, 0, 0])
    assert struct.unpack_from("<HHBBBBI", msgs[3], 8) == (0, 64, 52, 11, 0, 52, 1023)
    # fill value v2 without a value; contiguous layout v3 over the 24 data bytes
    assert msgs[5][:4] == bytes([2, 2, 2, 0])
    lv, lc, daddr, nbytes = struct.unpack_from("<BBQQ", msgs[8], 0)
    assert (lv, lc, nbytes) == (3, 1, 24)
    assert np.frombuffer(bytes(w.buf[daddr:daddr + 24]), "<f8").tolist() == [1.0, 2.0, 3.0]


def test_snapshot_file_structure(tmp_path):
    """The driver's file: root `t`, per grid x, y, t -> /t and the four (outputs, ny, nx) fields."""
    rng = np.random.default_rng(3)
    grids = [types.SimpleNamespace(x=rng.random((4, 6)), y=rng.random((4, 6))),
             types.SimpleNamespace(x=rng.random((5, 3)), y=rng.random((5, 3)))]
    frames = [[rng.random((4, 4, 6)), rng.random((4, 5, 3))] for _ in range(3)]
    path = str(tmp_path / "output.hdf")
    hdf5.write_snapshots(path, ["left", "right"], grids, [0, 10, 20], frames)
    tree = hdf5.read(path)
    assert sorted(tree) == ["left", "right", "t"]
    np.testing.assert_array_equal(tree["t"], np.array([0, 10, 20], np.uint64))
    for b, name in enumerate(["left", "right"]):
        g = tree[name]
        assert sorted(g) == ["e", "rho", "rhou", "rhov", "t", "x", "y"]
        assert g["t"].target == "/t"
        np.testing.assert_array_equal(g["x"], grids[b].x)
        for c, comp in enumerate(("rho", "rhou", "rhov", "e")):
            np.testing.assert_array_equal(g[comp], np.stack([f[b][c] for f in frames]))


def test_reader_rejects_truncation(tmp_path):
    path = str(tmp_path / "f.hdf")
    hdf5.write(path, {"t": np.arange(3, dtype=np.uint64)})
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-8])
    with pytest.raises(ValueError):
        hdf5.read(path)
