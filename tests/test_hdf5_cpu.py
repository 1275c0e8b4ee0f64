"""The HDF5 reader (cosmonpc_b200.hdf5) on files of the layouts it supports:
contiguous and chunked (shuffle + deflate) datasets of several element types
and byte orders in a symbol-table root group, written by the module's writer;
non-HDF5 input is refused."""
import numpy as np
import pytest


def test_columns_round_trip(tmp_path):
    from cosmonpc_b200 import hdf5

    rng = np.random.default_rng(4)
    n = 12345
    cols = {"x": rng.random(n) * 1000.0, "y": rng.random(n).astype(">f8"), "z": rng.random(n).astype(np.float32),
            "ID": np.arange(n, dtype=np.int64), "flag": (rng.random(n) < 0.5).astype(np.uint8),
            "k": rng.integers(-5, 5, n).astype(">i4"), "vx": rng.normal(0, 300, n)}
    path = hdf5.write_columns(str(tmp_path / "cat.h5"), cols, chunked={"vx": 1000, "z": 4096, "k": 777})
    infos, _ = hdf5.open_datasets(path)
    assert set(infos) == set(cols)
    assert infos["vx"].layout == "chunked" and infos["x"].layout == "contiguous"
    assert infos["y"].dtype.byteorder == ">" and infos["z"].dtype == np.float32
    for name, v in cols.items():
        got = hdf5.read_dataset(path, name)
        assert got.dtype == v.dtype, name
        np.testing.assert_array_equal(got, v)


def test_empty_and_single_chunk(tmp_path):
    from cosmonpc_b200 import hdf5

    path = hdf5.write_columns(str(tmp_path / "e.h5"), {"x": np.zeros(0), "y": np.arange(5.0)}, chunked={"y": 64})
    assert hdf5.read_dataset(path, "x").size == 0
    np.testing.assert_array_equal(hdf5.read_dataset(path, "y"), np.arange(5.0))


def test_not_hdf5(tmp_path):
    from cosmonpc_b200 import hdf5

    p = tmp_path / "x.h5"
    p.write_bytes(b"SIMPLE  = T" + b" " * 3000)
    with pytest.raises(ValueError):
        hdf5.open_datasets(str(p))
