"""The drivers' HDF5 output (cupf_b200/host/h5_writer.cpp; the reference writes
its QoIs and fields with h5write_1d, 3DgrainMPI/PhaseFieldCpu.cpp:584-613).

No libhdf5 or h5py exists in this environment, so the files are read back with
tests/h5read.py, a reader written separately from the writer after the
published format specification.  The reader itself is first checked on a file
written by libhdf5 (SciPy's MATLAB v7.3 test fixture, whose content SciPy's own
tests define as 0..2*pi in steps of pi/4).
"""
import os
import struct

import numpy as np
import pytest

from cupf_b200 import host_api
from tests.h5read import H5File

MAT73 = None
try:
    import scipy
    MAT73 = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data",
                         "testhdf5_7.4_GLNX86.mat")
except Exception:
    pass


@pytest.mark.skipif(MAT73 is None or not os.path.exists(MAT73), reason="SciPy test data absent")
def test_reader_reads_a_libhdf5_file():
    f = H5File(MAT73)
    assert f.keys() == ["testdouble"]
    v = f["testdouble"]
    assert v.dtype == np.float64 and v.shape == (9, 1)
    assert np.allclose(v.ravel(), np.arange(9) * np.pi / 4, rtol=0, atol=1e-15)


def test_roundtrip_reference_dataset_set(tmp_path):
    """The datasets OutputQoIs writes for a line run, with their dtypes."""
    rng = np.random.default_rng(0)
    arrays = {
        "x_coordinates": rng.random(66).astype(np.float32),
        "y_coordinates": rng.random(66).astype(np.float32),
        "z_coordinates": rng.random(300).astype(np.float32),
        "angles": rng.random(41).astype(np.float32),
        "r0": np.array([1.5], np.float32), "z0": np.array([0.25], np.float32),
        "x0": np.array([0.0], np.float32), "top": np.array([3.0], np.float32),
        "angle": np.array([0.0], np.float32), "V": np.array([0.0], np.float32),
        "fractions": rng.random(20 * 7).astype(np.float32),
        "tip_y": rng.integers(0, 100, 7).astype(np.int32),
        "cross_sec": rng.integers(0, 20, 64 * 64).astype(np.int32),
        "extra_area": rng.integers(-5, 5, 140).astype(np.int32),
        "total_area": rng.integers(0, 999, 140).astype(np.int32),
        "tip_final": np.array([88], np.int32),
        "node_region": np.zeros(0, np.int32),
    }
    p = str(tmp_path / "q.h5")
    host_api.h5_write(p, arrays)
    f = H5File(p)
    assert f.keys() == sorted(arrays)
    for k, v in arrays.items():
        got = f[k]
        assert got.dtype == v.dtype.newbyteorder("<") and got.shape == v.shape, k
        assert np.array_equal(got, v), k


def test_roundtrip_many_datasets_and_dtypes(tmp_path):
    """More names than one symbol-table node holds (32): several nodes under
    the B-tree; every supported element type; names in byte order."""
    rng = np.random.default_rng(1)
    arrays = {}
    for i in range(150):
        dt = [np.int8, np.int16, np.int32, np.int64, np.float32, np.float64][i % 6]
        n = int(rng.integers(0, 40))
        a = (rng.standard_normal(n) * 1000).astype(dt)
        arrays["d%03d_%s" % (149 - i, np.dtype(dt).name)] = a
    arrays["Z_upper"] = np.arange(5, dtype=np.int32)  # sorts before lower case
    p = str(tmp_path / "many.h5")
    host_api.h5_write(p, arrays)
    f = H5File(p)
    assert f.keys() == sorted(arrays)
    for k, v in arrays.items():
        assert np.array_equal(f[k], v), k


def test_structure_of_the_file(tmp_path):
    """Fields a libhdf5 reader checks first: signature, superblock version 0,
    8-byte offsets and lengths, end-of-file address = file size, root symbol
    table entry caching the B-tree and local heap, an empty heap free list
    encoded as 1, and the B-tree's keys bracketing every node's names."""
    p = str(tmp_path / "s.h5")
    names = ["alpha", "b", "c" * 40]
    host_api.h5_write(p, {k: np.arange(3, dtype=np.float32) for k in names})
    b = open(p, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert b[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    base, fs, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert (base, fs, drv) == (0, 2 ** 64 - 1, 2 ** 64 - 1) and eof == len(b)
    _, oh, cache, _, btree, heap = struct.unpack_from("<QQIIQQ", b, 56)
    assert cache == 1
    assert b[heap:heap + 4] == b"HEAP"
    dsize, free, daddr = struct.unpack_from("<QQQ", b, heap + 8)
    assert free == 1 and dsize % 8 == 0
    hd = b[daddr:daddr + dsize]
    assert b[btree:btree + 4] == b"TREE"
    used = struct.unpack_from("<H", b, btree + 6)[0]
    keys = [struct.unpack_from("<Q", b, btree + 24 + 16 * i)[0] for i in range(used + 1)]
    name_at = lambda o: hd[o:hd.index(b"\0", o)].decode()
    assert name_at(keys[0]) == "" and name_at(keys[-1]) == max(names)
    # the root object header carries the same addresses in its Symbol Table message
    assert b[oh] == 1
    mtype, msize = struct.unpack_from("<HH", b, oh + 16)
    assert (mtype, msize) == (0x11, 16)
    assert struct.unpack_from("<QQ", b, oh + 24) == (btree, heap)


def test_writer_rejects_bad_arguments(tmp_path):
    with pytest.raises(TypeError):
        host_api.h5_write(str(tmp_path / "x.h5"), {"u": np.arange(3, dtype=np.uint16)})
    with pytest.raises(IOError):
        host_api.h5_write(str(tmp_path / "no" / "such" / "dir.h5"), {"a": np.zeros(1, np.int32)})
