"""HDF5 files without libhdf5 (bfps_b200.h5): the reference's own fixture
read by its structure, and round trips of what the launcher writes
(parameters, checkpoints, growing statistics)."""
import os

import numpy as np
import pytest

from bfps_b200 import h5

FIXTURE = os.path.join(os.environ.get("BFPS_REFERENCE", "/root/reference"), "bfps", "test",
                       "B32p1e4_checkpoint_0.h5")


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="reference checkout absent")
def test_reads_reference_fixture_by_structure(golden):
    """bfps/test/B32p1e4_checkpoint_0.h5 (written by libhdf5 through h5py and
    the reference's C++ writers) read through its groups, not offsets."""
    with h5.File(FIXTURE) as f:
        assert f.keys() == ["tracers0", "vorticity"]
        assert f["vorticity/complex"].keys() == ["0", "32", "64"]
        assert f["tracers0/rhs"].keys() == ["0", "32", "64"]
        for it in (0, 32, 64):
            v = f["vorticity/complex/%d" % it]
            assert v.shape == (32, 32, 17, 3) and v.dtype == np.complex64
            assert np.array_equal(v[()], golden["vorticity_%d" % it])
        nk = golden["state_32"].shape[0]
        for it in (32, 64):
            assert np.array_equal(f["tracers0/state/%d" % it][()][:nk], golden["state_%d" % it])
            assert np.array_equal(f["tracers0/rhs/%d" % it][()][:, :nk], golden["rhs_%d" % it])
        np.random.seed(2)
        assert np.array_equal(f["tracers0/state/0"][()], np.random.random((10000, 3)) * 2 * np.pi)


def test_round_trip_types(tmp_path):
    p = str(tmp_path / "a.h5")
    rng = np.random.default_rng(0)
    data = {
        "vorticity/complex/0": (rng.standard_normal((8, 8, 5, 3)) + 1j * rng.standard_normal((8, 8, 5, 3))).astype(np.complex64),
        "vorticity/complex/16": (rng.standard_normal((8, 8, 5, 3)) * 1j).astype(np.complex128),
        "tracers0/state/0": rng.random((100, 3)),
        "tracers0/rhs/0": np.zeros((4, 100, 3)),
        "kspace/nshell": np.arange(7, dtype=np.int64),
        "kspace/kshell": rng.random(7).astype(np.float32),
        "parameters/nx": np.int64(32),
        "parameters/nu": np.float64(0.0625),
        "parameters/forcing_type": np.bytes_(b"linear"),
        "iteration": np.int32(64),
    }
    with h5.File(p, "w") as f:
        for k, v in data.items():
            f[k] = v
    with h5.File(p) as f:
        assert f.keys() == ["iteration", "kspace", "parameters", "tracers0", "vorticity"]
        for k, v in data.items():
            a = f[k][()]
            assert a.dtype == np.asarray(v).dtype, k
            assert np.array_equal(a, v), k
        assert f["parameters/forcing_type"][()] == b"linear"


def test_append_many_links(tmp_path):
    """Groups beyond one symbol-table node, grown over several sessions."""
    p = str(tmp_path / "b.h5")
    with h5.File(p, "w") as f:
        f.create_group("tracers0/velocity")
    for start in range(0, 300, 100):
        with h5.File(p, "a") as f:
            for i in range(start, start + 100):
                f["tracers0/velocity/%d" % i] = np.full((1, 5, 3), float(i))
    with h5.File(p, "r") as f:
        keys = f["tracers0/velocity"].keys()
        assert sorted(int(k) for k in keys) == list(range(300))
        for i in (0, 127, 128, 255, 299):
            assert np.all(f["tracers0/velocity/%d" % i][()] == i)
    with pytest.raises(h5.H5Error):
        with h5.File(p, "a") as f:
            f["tracers0/velocity/7"] = np.zeros(3)


def test_growing_chunked_statistics(tmp_path):
    """statistics/* datasets: created (1, ...) with an unlimited first axis,
    grown a row per statistics step across chunks (hdf5_tools.cpp:74-92)."""
    p = str(tmp_path / "c.h5")
    with h5.File(p, "w") as f:
        f.create_dataset("statistics/moments/velocity", (1, 10, 4), chunks=(3, 10, 4),
                         maxshape=(None, 10, 4), dtype=np.float64)
        f.create_dataset("statistics/histograms/velocity", (1, 16, 4), chunks=(5, 16, 4),
                         maxshape=(None, 16, 4), dtype=np.int64)
    rows = np.arange(11 * 40, dtype=np.float64).reshape(11, 10, 4)
    hist = np.arange(11 * 64, dtype=np.int64).reshape(11, 16, 4)
    for t in range(11):
        with h5.File(p, "a") as f:
            f["statistics/moments/velocity"].write_rows(t, rows[t:t + 1])
            f["statistics/histograms/velocity"].write_rows(t, hist[t:t + 1])
    with h5.File(p) as f:
        m = f["statistics/moments/velocity"]
        assert m.shape == (11, 10, 4) and m.maxshape == (None, 10, 4) and m.chunks == (3, 10, 4)
        assert np.array_equal(m[()], rows)
        assert np.array_equal(f["statistics/histograms/velocity"][()], hist)
        assert np.array_equal(m[4:6], rows[4:6])
    with h5.File(p, "a") as f:
        f["statistics/moments/velocity"].resize(20)
    with h5.File(p) as f:
        a = f["statistics/moments/velocity"][()]
        assert a.shape == (20, 10, 4) and np.array_equal(a[:11], rows) and not a[11:].any()


def test_rejects_what_it_does_not_read(tmp_path):
    p = str(tmp_path / "d.h5")
    open(p, "wb").write(b"not hdf5" * 20)
    with pytest.raises(h5.H5Error):
        h5.File(p)
    with pytest.raises(FileNotFoundError):
        h5.File(str(tmp_path / "missing.h5"))
    q = str(tmp_path / "e.h5")
    with h5.File(q, "w") as f:
        f["x"] = np.zeros(3)
    with h5.File(q, "r") as f:
        with pytest.raises(h5.H5Error):
            f["y"] = np.zeros(3)


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="reference checkout absent")
def test_append_to_reference_written_file(tmp_path, golden):
    """Adding a checkpoint to a libhdf5-written file: the parent entries that
    cache a group's B-tree and heap (cache type 1, as libhdf5 writes them)
    must not keep the old addresses."""
    import shutil
    p = str(tmp_path / "cp.h5")
    shutil.copy(FIXTURE, p)
    os.chmod(p, 0o644)
    with h5.File(p) as f:
        cached = set()
        f._group_links(f._lookup("/"), cached)
        assert cached == {"tracers0", "vorticity"}   # libhdf5 caches group entries
    with h5.File(p, "a") as f:
        f["vorticity/complex/96"] = golden["vorticity_64"]
        f["tracers0/state/96"] = np.ones((10, 3))
    with h5.File(p) as f:
        assert f["vorticity/complex"].keys() == ["0", "32", "64", "96"]
        assert np.array_equal(f["vorticity/complex/96"][()], golden["vorticity_64"])
        assert np.array_equal(f["vorticity/complex/32"][()], golden["vorticity_32"])
        assert f["tracers0/state"].keys() == ["0", "32", "64", "96"]
        # every group on the modified paths was rewritten without caches,
        # so no entry points at the groups' old B-trees and heaps
        for gpath in ("/", "/vorticity", "/tracers0"):
            cached = set()
            f._group_links(f._lookup(gpath), cached)
            assert cached == set(), gpath


def test_variable_length_strings(tmp_path):
    """h5py writes Python str values (bfps_info/*) as variable-length
    strings in a global heap collection: datatype class 9, elements of
    (length, collection address, object index)."""
    import struct
    p = str(tmp_path / "v.h5")
    words = [b"linear", b"NSVEparticles-single", b""]
    with h5.File(p, "w") as f:
        # a global heap collection holding the strings (objects 1..3)
        body = b""
        for i, w in enumerate(words, 1):
            body += struct.pack("<HH4xQ", i, 1, len(w)) + w + b"\0" * ((-len(w)) % 8)
        size = 16 + len(body) + 16
        size = max(size, 4096)
        coll = b"GCOL" + bytes([1, 0, 0, 0]) + struct.pack("<Q", size) + body
        coll += struct.pack("<HH4xQ", 0, 0, size - 16 - len(body) - 16) + b"\0" * (size - len(coll) - 16)
        gaddr = f._append(coll)
        # a 1-D dataset of three vlen strings: class 9 (version 1), string
        # type, base type a one-byte unsigned integer
        base = struct.pack("<B3sI", 0x10, (0).to_bytes(3, "little"), 1) + struct.pack("<HH", 0, 8)
        dtype = struct.pack("<B3sI", 0x19, (1).to_bytes(3, "little"), 16) + base
        elems = b"".join(struct.pack("<IQI", len(w), gaddr, i) for i, w in enumerate(words, 1))
        data = f._append(elems)
        layout = struct.pack("<BBQQ", 3, 1, data, len(elems))
        hdr = f._write_object_header([(h5.MSG_DATASPACE, f._dataspace((3,), (3,))),
                                      (h5.MSG_DATATYPE, dtype, 1), (h5.MSG_LAYOUT, layout, 1)])
        f._link("/bfps_info/strings", hdr)
    with h5.File(p) as f:
        got = f["bfps_info/strings"][()]
        assert list(got) == ["linear", "NSVEparticles-single", ""]
