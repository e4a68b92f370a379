"""Autotuner cache on the CPU: entries put through the C ABI land in a JSON
file (a valid JSON document, rewritten through a temporary file), survive a
clear + reload, and are looked up by (routine, flags, sizes, precision)."""
import json
import os

import pytest

import TensorBLAS as TB


@pytest.fixture()
def cache(tmp_path):
    path = str(tmp_path / "tune.json")
    TB.autotune_set_file(path)
    TB.lib.tb_autotune_clear()
    yield path
    TB.lib.tb_autotune_clear()
    TB.autotune_set_file(None)


def test_put_get_file_roundtrip(cache):
    assert TB.autotune_entries() == 0
    TB._check(TB.lib.tb_autotune_put(b"strsm", b"L", 16384, 16384, TB.PLAIN, 256, 1, 6.1))
    TB._check(TB.lib.tb_autotune_put(b"ssyrk", b"LN", 4096, 4096, TB.SPLIT, 256, 0, 0.4))
    assert TB.autotune_entries() == 2
    assert TB.autotune_get("strsm", "L", 16384, 16384, TB.PLAIN) == (256, 1)
    assert TB.autotune_get("ssyrk", "LN", 4096, 4096, TB.SPLIT) == (256, 0)
    assert TB.autotune_get("ssyrk", "LN", 4096, 4096, TB.PLAIN) is None  # precision is part of the key
    doc = json.load(open(cache))
    assert doc["format"] == "tensorblas-autotune-1"
    assert len(doc["entries"]) == 2
    keys = sorted(e["key"] for e in doc["entries"])
    assert keys[0].split("|")[1:] == ["ssyrk", "LN", "4096", "4096", "1"]
    assert not [f for f in os.listdir(os.path.dirname(cache)) if ".tmp." in f]
    TB.lib.tb_autotune_clear()
    assert TB.autotune_entries() == 0
    TB.autotune_set_file(cache)  # reload
    assert TB.autotune_entries() == 2
    assert TB.autotune_get("strsm", "L", 16384, 16384, TB.PLAIN) == (256, 1)


def test_put_rejects_bad_entries(cache):
    assert TB.lib.tb_autotune_put(b"strsm", b"L", 8, 8, 0, 0, 1, 1.0) == 1   # nb <= 0
    assert TB.lib.tb_autotune_put(b"strsm", b"L", 8, 8, 0, 128, 3, 1.0) == 1  # engine not 0 / 1 / 2
    assert TB.lib.tb_autotune_put(b"strsm", b"L", 8, 8, 0, 128, -1, 1.0) == 1
    assert TB.autotune_entries() == 0


def test_narrow_engine_entries_roundtrip(cache):
    """Engine 2 (single-CTA 128 x 128 tiles for the plain launches) is a
    valid entry and survives the file round trip."""
    TB._check(TB.lib.tb_autotune_put(b"ssyr2k", b"LN", 1024, 8192, TB.PLAIN, 256, 2, 0.08))
    TB._check(TB.lib.tb_autotune_put_ex(b"strmm", b"U", 4096, 256, TB.PLAIN, 256, 2, 1, 0.05))
    TB.lib.tb_autotune_clear()
    TB.autotune_set_file(cache)  # reload
    assert TB.autotune_get("ssyr2k", "LN", 1024, 8192, TB.PLAIN) == (256, 2)
    assert TB.autotune_get_ex("strmm", "U", 4096, 256, TB.PLAIN) == (256, 2, 1)


def test_splitk_entries_roundtrip_and_old_format(cache):
    TB._check(TB.lib.tb_autotune_put_ex(b"ssyrk", b"LN", 1024, 16384, TB.PLAIN, 256, 0, 8, 0.05))
    assert TB.autotune_get_ex("ssyrk", "LN", 1024, 16384, TB.PLAIN) == (256, 0, 8)
    assert TB.autotune_get("ssyrk", "LN", 1024, 16384, TB.PLAIN) == (256, 0)
    assert TB.lib.tb_autotune_put_ex(b"ssyrk", b"LN", 8, 8, 0, 256, 0, 0, 1.0) == 1  # split-K count < 1
    doc = json.load(open(cache))
    assert [e["splitk"] for e in doc["entries"]] == [8]
    # a file written before the split-K field existed still loads (one pass)
    key = doc["entries"][0]["key"].replace("|1024|", "|2048|")
    with open(cache, "w") as f:
        f.write('{\n "format": "tensorblas-autotune-1",\n "entries": [\n'
                f'  {{"key": "{key}", "nb": 256, "engine": 1, "ms": 0.5}}\n ]\n}}\n')
    TB.lib.tb_autotune_clear()
    TB.autotune_set_file(cache)
    assert TB.autotune_get_ex("ssyrk", "LN", 2048, 16384, TB.PLAIN) == (256, 1, 1)
