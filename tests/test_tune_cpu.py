"""The autotuner's table without a GPU: JSON load, dump, save, clear, mode
switching, and rejection of malformed files."""

import json

import pytest

from cucim_b200 import _lib, tune

TABLE = {"format": "cimx-tune-1", "entries": [
    {"device": "NVIDIA B200 (148 SMs)", "key": "H>f [512,1024,1024] a0k9o4m1z a1k17o8m1z "
     "a2k17o8m1z t0", "flags": 64, "ms": 1.5, "candidates": [[0, 1.6], [64, 1.5]]},
    {"device": 'other "quoted" device', "key": "f>f [2048,2048] a0k33o16m0c a1k33o16m0c t4",
     "flags": 4, "ms": 0.02, "candidates": []},
]}


@pytest.fixture
def clean():
    tune.clear()
    yield
    tune.clear()


def test_load_dump_save_roundtrip(tmp_path, clean):
    p = tmp_path / "t.json"
    p.write_text(json.dumps(TABLE))
    tune.load(p)
    got = {(e["device"], e["key"]): e for e in tune.entries()}
    assert len(got) == 2
    e = got[("NVIDIA B200 (148 SMs)", TABLE["entries"][0]["key"])]
    assert e["flags"] == 64 and e["ms"] == 1.5 and e["candidates"] == [[0, 1.6], [64, 1.5]]
    assert ('other "quoted" device', TABLE["entries"][1]["key"]) in got
    q = tmp_path / "saved.json"
    tune.save(q)
    tune.clear()
    assert tune.entries() == []
    tune.load(q)
    assert {(e["device"], e["key"]) for e in tune.entries()} == set(got)


def test_malformed_tables_are_rejected(tmp_path, clean):
    for text in ("[]", "{\"format\": \"other\", \"entries\": []}", "{\"format\": \"cimx-tune-1\"}",
                 "{\"format\": \"cimx-tune-1\", \"entries\": [{\"key\": \"k\"}]}", "{not json"):
        p = tmp_path / "bad.json"
        p.write_text(text)
        with pytest.raises(RuntimeError):
            tune.load(p)
    with pytest.raises(RuntimeError):
        tune.load(tmp_path / "missing.json")


def test_mode_switching():
    prev = tune.mode()
    assert prev in (tune.OFF, tune.USE, tune.ON)
    with tune.tuning(tune.OFF):
        assert tune.mode() == tune.OFF
    assert tune.mode() == prev
    assert _lib.lib.cimx_tune_mode(7) == _lib.E_INVALID
