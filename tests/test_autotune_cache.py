"""Host logic of the autotuner's JSON cache (no GPU): round trip, a corrupt
file read as empty, and an unwritable location costing only re-tuning."""

import json
import os
import stat

from finitevolx_b200 import autotune


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("FVX_AUTOTUNE_CACHE", str(path))
    assert autotune._load() == {}
    autotune._store("qg_stage/dev/weno5/2048", {"tile": "64x32", "ms": [1.0, 2.0]})
    autotune._store("dst_kernel/dev/2048", {"kernel": "single64"})
    data = json.loads(path.read_text())
    assert data["qg_stage/dev/weno5/2048"]["tile"] == "64x32"
    assert autotune._load() == data


def test_corrupt_cache_reads_as_empty(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    path.write_text("{not json")
    monkeypatch.setenv("FVX_AUTOTUNE_CACHE", str(path))
    assert autotune._load() == {}
    autotune._store("k", 1)  # overwrites the corrupt file
    assert autotune._load() == {"k": 1}


def test_unwritable_cache_is_ignored(tmp_path, monkeypatch):
    ro = tmp_path / "ro"
    ro.mkdir()
    ro.chmod(stat.S_IRUSR | stat.S_IXUSR)
    monkeypatch.setenv("FVX_AUTOTUNE_CACHE", str(ro / "deeper" / "tune.json"))
    try:
        autotune._store("k", 1)  # must not raise
        if os.geteuid() != 0:  # root can write anyway
            assert autotune._load() == {}
    finally:
        ro.chmod(stat.S_IRWXU)
