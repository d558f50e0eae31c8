"""CPU: the Zarr v3 layout written for QG snapshots (metadata and raw
little-endian chunks) reads back exactly, and matches the v3 array-metadata
fields an xarray / zarr 3 reader needs."""

import json

import numpy as np

from finitevolx_b200.snapshots import _array_meta, _write_chunk, _write_json, read_zarr_v3, write_array


def test_zarr_v3_roundtrip(tmp_path):
    root = tmp_path / "run.zarr"
    rng = np.random.default_rng(0)
    data = rng.standard_normal((3, 5, 7)).astype(np.float32)
    _write_json(root / "zarr.json", {"zarr_format": 3, "node_type": "group", "attributes": {"model": "qg"}})
    _write_json(root / "q" / "zarr.json",
                _array_meta(data.shape, (1, 5, 7), data.dtype, ("time", "y", "x"), {"units": "s-1"}))
    for t in range(3):
        _write_chunk(root, "q", (t, 0, 0), data[t])
    write_array(root, "time", np.array([0.0, 10.0, 20.0]), ("time",), {"units": "s"})
    got = read_zarr_v3(root)
    assert got["__attrs__"] == {"model": "qg"}
    arr, dims, attrs = got["q"]
    assert arr.dtype == np.float32 and dims == ["time", "y", "x"] and attrs == {"units": "s-1"}
    np.testing.assert_array_equal(arr, data)
    np.testing.assert_array_equal(got["time"][0], [0.0, 10.0, 20.0])
    meta = json.loads((root / "q" / "zarr.json").read_text())
    assert meta["zarr_format"] == 3 and meta["node_type"] == "array"
    assert meta["chunk_key_encoding"] == {"name": "default", "configuration": {"separator": "/"}}
    assert meta["codecs"] == [{"name": "bytes", "configuration": {"endian": "little"}}]
    assert (root / "q" / "c" / "2" / "0" / "0").stat().st_size == 5 * 7 * 4


def test_missing_chunks_read_as_fill(tmp_path):
    root = tmp_path / "s.zarr"
    _write_json(root / "zarr.json", {"zarr_format": 3, "node_type": "group", "attributes": {}})
    _write_json(root / "a" / "zarr.json", _array_meta((2, 3), (1, 3), np.dtype("float64"), ("t", "x"), {}))
    _write_chunk(root, "a", (1, 0), np.arange(3.0))
    arr = read_zarr_v3(root)["a"][0]
    assert np.isnan(arr[0]).all() and np.array_equal(arr[1], np.arange(3.0))
