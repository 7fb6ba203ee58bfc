"""The HDF5 layer of the output files (inchman_b200.h5) and the reference's file
layout (DiffusionModel.cpp:934-1296, InchmanDiffusionModel.cpp:240-274,
doc/source/hdf5.rst), on the CPU.

The reader is first checked on a file that libhdf5 itself wrote (scipy ships one as
test data: a MATLAB 7.3 file, superblock version 0 behind a 512-byte user block);
the writer is then checked through the reader and against the format's fixed
structures byte by byte."""
import os
import struct

import numpy as np
import pytest

from inchman_b200 import h5

HERE = os.path.dirname(__file__)


def _libhdf5_sample():
    try:
        import scipy.io.matlab as mio
    except ImportError:
        return None
    p = os.path.join(os.path.dirname(mio.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    return p if os.path.exists(p) else None


def test_reader_reads_a_file_written_by_libhdf5():
    p = _libhdf5_sample()
    if p is None:
        pytest.skip("scipy's HDF5 test file is not installed")
    root = h5.read(p)
    assert list(root) == ["testdouble"]
    d = root["testdouble"]
    assert d.value.dtype == np.float64 and d.value.shape == (9, 1)
    assert np.allclose(d.value.ravel(), np.pi / 4 * np.arange(9))
    assert d.attrs["MATLAB_class"] == "double"


def _tree(ndump=300, nruns=12):
    g = h5.Group()
    m = g.create_group("Model")
    m.attrs["numSpecies"] = np.array([2], np.int32)
    m.attrs["numRuns"] = np.array([nruns], np.int32)
    m.create_dataset("Species", ["A", "Bee"])
    m.create_dataset("InchmanFile", "<sbml>text</sbml>")
    c = m.create_group("Compartments")
    c.create_dataset("World", np.array([0, 0, 31, 31], np.int32))
    runs = g.create_group("Runs")
    for r in range(nruns):
        rg = runs.create_group(str(r))
        for t in range(ndump):
            dg = rg.create_group(f"Dump_{t}")
            dg.attrs["time"] = np.array([t], np.float32)
            dg.create_dataset("A", np.arange(20, dtype=np.int32).reshape(4, 5) + 1000 * r + t)
            dg.create_dataset("Bee", np.full((4, 5), t / 7, np.float32))
            dg.create_group("Individuals")
    g.create_dataset("u64", np.arange(5, dtype=np.uint64) << 40)
    g.create_dataset("f64", np.linspace(0, 1, 7))
    return g


def test_round_trip(tmp_path):
    path = str(tmp_path / "t.h5")
    h5.write(path, _tree())
    r = h5.read(path)
    assert r["Model"].attrs["numRuns"].tolist() == [12]
    assert r["Model/Species"].value == ["A", "Bee"]
    assert r["Model/InchmanFile"].value == "<sbml>text</sbml>"
    assert r["Model/Compartments/World"].value.tolist() == [0, 0, 31, 31]
    # groups list their members sorted by name (lexical: "10" before "2")
    assert list(r["Runs"]) == sorted(str(i) for i in range(12))
    dumps = list(r["Runs/7"])
    assert len(dumps) == 300 and dumps[:4] == ["Dump_0", "Dump_1", "Dump_10", "Dump_100"]
    d = r["Runs/7/Dump_123"]
    assert d.attrs["time"].dtype == np.float32 and d.attrs["time"].tolist() == [123.0]
    assert np.array_equal(d["A"].value, np.arange(20, dtype=np.int32).reshape(4, 5) + 7123)
    assert d["Bee"].value.dtype == np.float32 and np.all(d["Bee"].value == np.float32(123 / 7))
    assert list(d["Individuals"]) == []
    assert np.array_equal(r["u64"].value, np.arange(5, dtype=np.uint64) << 40)
    assert np.array_equal(r["f64"].value, np.linspace(0, 1, 7))


def test_fixed_structures(tmp_path):
    """Superblock version 0 with 8-byte offsets, the default node sizes, and every
    group's B-tree / symbol table nodes / local heap where the root entry and the
    symbol table messages point."""
    path = str(tmp_path / "t.h5")
    h5.write(path, _tree(ndump=40, nruns=2))
    b = open(path, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert b[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    leaf_k, node_k, flags = struct.unpack_from("<HHI", b, 16)
    assert (leaf_k, node_k, flags) == (4, 16, 0)
    base, free, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert base == 0 and free == h5.UNDEF and drv == h5.UNDEF and eof == len(b)
    name_off, oh, cache, _, bt, heap = struct.unpack_from("<QQIIQQ", b, 56)
    assert cache == 1 and b[bt:bt + 4] == b"TREE" and b[heap:heap + 4] == b"HEAP"
    assert b[oh] == 1                                   # version 1 object header
    nmsg, _, size = struct.unpack_from("<HII", b, oh + 2)
    t, s, fl = struct.unpack_from("<HHB", b, oh + 16)
    assert t == 0x11 and s == 16
    assert struct.unpack_from("<QQ", b, oh + 24) == (bt, heap)
    # local heap: "" at offset 0, a free block at the end whose next pointer is 1
    dsize, free_head, seg = struct.unpack_from("<QQQ", b, heap + 8)
    assert b[seg:seg + 8] == b"\0" * 8
    assert struct.unpack_from("<QQ", b, seg + free_head) == (1, dsize - free_head)
    # every B-tree node: full size, children in range, keys name offsets in the heap
    ntype, level, used, left, right = struct.unpack_from("<BBHQQ", b, bt + 4)
    assert ntype == 0 and level == 0 and left == h5.UNDEF and right == h5.UNDEF
    snod = struct.unpack_from("<Q", b, bt + 32)[0]
    assert b[snod:snod + 8] == b"SNOD" + bytes([1, 0]) + struct.pack("<H", 4)   # Model, Runs, f64, u64


def test_symbol_table_nodes_are_sorted_and_full_sized(tmp_path):
    path = str(tmp_path / "t.h5")
    g = h5.Group()
    names = [f"n{i:03d}" for i in range(50)][::-1]
    for nm in names:
        g.create_group(nm)
    h5.write(path, g)
    b = open(path, "rb").read()
    _, _, _, _, bt, heap = struct.unpack_from("<QQIIQQ", b, 56)
    _, level, used = struct.unpack_from("<BBH", b, bt + 4)
    assert level == 0 and used == 7                      # 50 names, 8 per node
    _, _, seg = struct.unpack_from("<QQQ", b, heap + 8)
    got = []
    for c in range(used):
        child = struct.unpack_from("<Q", b, bt + 32 + 16 * c)[0]
        n = struct.unpack_from("<H", b, child + 6)[0]
        for e in range(n):
            off = struct.unpack_from("<Q", b, child + 8 + 40 * e)[0]
            got.append(b[seg + off:b.index(b"\0", seg + off)].decode())
        # the key after child c is the last name in it
        key = struct.unpack_from("<Q", b, bt + 32 + 16 * c + 8)[0]
        assert b[seg + key:b.index(b"\0", seg + key)].decode() == got[-1]
    assert got == sorted(names)


def test_reference_layout_from_a_model_file(tmp_path):
    """The output tree of the CLI for synthetic snapshots of a fixture model: the
    groups, attributes, datasets and dump names of the reference's writer."""
    from inchman_b200 import cli, sbml
    lm = sbml.load(os.path.join(HERE, "golden", "models", "ab_drift.xml"), overrides={"k2": 0.25})
    m = lm.model
    n, R = 4, 3
    snaps = np.arange(n * R * m.num_species * m.height * m.width, dtype=np.int32).reshape(
        n, R, m.num_species, m.height, m.width)
    times = np.array([0.0, 0.1, 0.2, 0.3], np.float32)
    times[2] = np.float32(0.1) + np.float32(0.1)
    path = str(tmp_path / "out.h5")
    h5.write(path, cli.output_tree(lm, snaps, times))
    f = h5.read(path)
    # read as python/gpgmp/io.py:read_gmp_hdf5 does
    model = f["Model"]
    assert model.attrs["numRuns"][0] == R and model.attrs["numSpecies"][0] == m.num_species
    species = model["Species"].value
    assert species == [s.id for s in m.species]
    assert model["InchmanFile"].value == lm.source
    assert set(model["Compartments"].children) == set(lm.compartments)
    assert f["Parameters"].attrs["k2"].tolist() == [np.float32(0.25)]
    first = f["Runs/0"]
    assert "Dump_0" in first
    assert list(first) == sorted(cli.dump_name(t) for t in times)
    assert cli.dump_name(np.float32(0.1)) == "Dump_0.100000001"
    assert cli.dump_name(np.float32(0.3)) == "Dump_0.300000012"
    for r in range(R):
        for k in range(n):
            d = f[f"Runs/{r}/{cli.dump_name(times[k])}"]
            assert d.attrs["time"][0] == times[k]
            for s, sid in enumerate(species):
                v = d[sid].value
                assert v.shape == (m.width, m.height) and v.dtype == np.int32
                assert np.array_equal(v.reshape(-1), snaps[k, r, s].reshape(-1))
            assert list(d["Individuals"]) == []


def test_cli_rejects_malformed_overrides(capsys):
    from inchman_b200 import cli
    with pytest.raises(SystemExit):
        cli.main([os.path.join(HERE, "golden", "models", "ab_drift.xml"), "--p", "k2"])
