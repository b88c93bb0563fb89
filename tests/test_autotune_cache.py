"""The autotuner's on-disk cache (host logic, no GPU): round trip, a corrupt file and an
unwritable location are tolerated, and the candidate lists stay within what the plan
accepts."""

import json
import os

from pyfourier_b200 import _autotune


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "autotune.json"
    monkeypatch.setenv("PYFOURIER_B200_CACHE", str(path))
    assert _autotune.cache_path() == str(path)
    assert _autotune._load_cache() == {}
    entry = {"B200|d3|os250x250x250|w4x4x4|m2^23|f1|b32|c1|l1": {"tile": [8, 8, 8], "chunk": 2048}}
    _autotune._save_cache(entry)
    assert json.loads(path.read_text()) == entry
    assert _autotune._load_cache() == entry
    assert not [p for p in os.listdir(path.parent) if p.endswith(".tmp")]  # written by rename


def test_corrupt_cache_reads_as_empty(tmp_path, monkeypatch):
    path = tmp_path / "autotune.json"
    path.write_text("{ not json")
    monkeypatch.setenv("PYFOURIER_B200_CACHE", str(path))
    assert _autotune._load_cache() == {}


def test_unwritable_cache_is_ignored(tmp_path, monkeypatch):
    blocker = tmp_path / "file"
    blocker.write_text("x")
    # the cache's directory would have to be created under a regular file
    monkeypatch.setenv("PYFOURIER_B200_CACHE", str(blocker / "autotune.json"))
    _autotune._save_cache({"k": 1})  # no exception
    assert _autotune._load_cache() == {}


def test_default_candidates():
    for ndim in (1, 2, 3):
        tiles, chunks = _autotune.default_candidates(ndim)
        assert tiles and all(len(t) == ndim and all(e >= 1 for e in t) for t in tiles)
        assert chunks and all(1 <= c <= 16384 for c in chunks)  # pfb_plan_set_chunk's range
