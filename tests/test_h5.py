"""diablo_b200.h5, the HDF5 writer and reader of the output files, on the
CPU: it reads a file the HDF5 library wrote (the reference's KH_test/grid.h5,
a committed fixture) and reads back what it writes, structure, types and
attributes included."""
import os
import struct

import numpy as np
import pytest

from diablo_b200 import h5

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_reads_the_reference_grid_file():
    t = h5.read(os.path.join(GOLDEN, "KH_test_grid.h5"))
    y = t.children["grids"].children["y"].data
    assert y.dtype == np.dtype("<f8") and y.shape == (66,)
    assert np.array_equal(y, np.loadtxt(os.path.join(GOLDEN, "kh_grid_y.txt")))


def test_round_trip_of_every_supported_form(tmp_path):
    rng = np.random.default_rng(3)
    root = h5.Group()
    root.attrs["Resolution"] = np.array([64, 65, 64], dtype=np.int32)
    root.attrs["Date"] = np.frombuffer(b"2026-12-04 01:00:00 ", dtype="S1")
    root.attrs["Info"] = "text"
    ts = root.group("Timestep")
    ts.attrs["Time"] = np.float64(1.5)
    ts.children["U"] = h5.Dataset(rng.standard_normal((5, 4, 3)))
    ts.children["F32"] = h5.Dataset(rng.standard_normal(7).astype(np.float32))
    ts.children["I64"] = h5.Dataset(np.arange(6, dtype=np.int64).reshape(2, 3), {"n": np.int32(-4)})
    ts.children["empty"] = h5.Dataset(np.zeros((0,)))
    deep = root.group("a").group("b").group("c")
    deep.children["s"] = h5.Dataset(np.float64(2.25))               # scalar dataset
    many = root.group("many")
    for i in range(300):                                            # beyond one default node
        many.children[f"{i:04d}"] = h5.Dataset(np.full(3, float(i)), {"Time": np.float64(0.1 * i)})
    path = str(tmp_path / "t.h5")
    h5.write(path, root)
    assert h5.is_hdf5(path)
    r = h5.read(path)
    assert list(r.attrs["Resolution"]) == [64, 65, 64] and r.attrs["Resolution"].dtype == np.int32
    assert r.attrs["Date"].tobytes() == b"2026-12-04 01:00:00 " and r.attrs["Info"].item() == b"text"
    t = r.children["Timestep"]
    assert t.attrs["Time"].shape == () and float(t.attrs["Time"]) == 1.5
    for k in ("U", "F32", "I64", "empty"):
        a, b = t.children[k].data, ts.children[k].data
        assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b), k
    assert int(t.children["I64"].attrs["n"]) == -4
    assert float(r.children["a"].children["b"].children["c"].children["s"].data) == 2.25
    m = r.children["many"].children
    assert len(m) == 300 and m["0299"].data[0] == 299.0 and float(m["0137"].attrs["Time"]) == pytest.approx(13.7)


def test_file_structure_is_the_library_default_layout(tmp_path):
    """Superblock version 0 with 8-byte offsets and lengths, the root group a
    version-1 object header whose message is a symbol table (B-tree and local
    heap), as the HDF5 1.8 library writes by default (and as the reference's
    grid.h5 is)."""
    root = h5.Group()
    root.group("g").children["d"] = h5.Dataset(np.arange(3.0))
    path = str(tmp_path / "s.h5")
    h5.write(path, root)
    for f in (path, os.path.join(GOLDEN, "KH_test_grid.h5")):
        b = open(f, "rb").read()
        assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8] == 0 and b[13] == 8 and b[14] == 8
        eof = struct.unpack_from("<Q", b, 40)[0]
        assert eof == len(b)
        oh = struct.unpack_from("<Q", b, 64)[0]
        assert b[oh] == 1                                           # object header version 1
        cache, = struct.unpack_from("<I", b, 72)
        bt, heap = struct.unpack_from("<QQ", b, 80)
        assert cache == 1 and b[bt:bt + 4] == b"TREE" and b[heap:heap + 4] == b"HEAP"


def test_rejects_what_it_does_not_handle(tmp_path):
    p = str(tmp_path / "x.h5")
    with open(p, "wb") as f:
        f.write(b"not hdf5 at all")
    assert not h5.is_hdf5(p)
    with pytest.raises(ValueError):
        h5.read(p)
    with pytest.raises(TypeError):
        h5.write(str(tmp_path / "y.h5"), h5.Group(children={"c": h5.Dataset(np.array([1 + 2j]))}))
