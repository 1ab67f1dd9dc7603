"""The persisted autotune table (frg_autotune_table_*): host-side behaviour.

The table maps (P, flux, dissipation form, geometry) to a tile variant of the
2D stage kernels.  These checks need no GPU: setting and reading entries,
the JSON round trip, rejection of malformed files and unknown variants, and
the committed B200 table itself.  tests/test_gpu_batch.py checks on the GPU
that a table entry changes the variant a new solve and a batched group use.
"""
import json
import os

import pytest

from frforge_b200 import _lib as L
from frforge_b200 import autotune as T


@pytest.fixture(autouse=True)
def empty_table():
    T.clear()
    yield
    T.clear()


def test_set_get_and_absent_key():
    assert T.get_variant(3, "hllc", "br0", False) is None
    T.set_variant(3, "hllc", "br0", False, 2)
    assert T.get_variant(3, "hllc", "br0", False) == 2
    assert T.get_variant(3, "hllc", "br0", True) is None  # curved is another key
    assert T.size() == 1


def test_unknown_variant_or_key_is_rejected():
    with pytest.raises(ValueError):
        T.set_variant(3, "hllc", "br0", False, 99)
    with pytest.raises(ValueError):
        T.set_variant(9, "hllc", "br0", False, 0)
    assert T.size() == 0


def test_json_round_trip(tmp_path):
    T.set_variant(1, "rusanov", "none", False, 1)
    T.set_variant(3, "hllc", "br0", False, 2)
    T.set_variant(5, "hllc", "local_dd", True, 1)
    path = str(tmp_path / "table.json")
    T.save(path)
    with open(path) as f:
        d = json.load(f)  # the file is plain JSON
    assert len(d["entries"]) == 3
    T.clear()
    assert T.size() == 0
    T.load(path)
    assert T.size() == 3
    assert T.get_variant(1, "rusanov", "none", False) == 1
    assert T.get_variant(3, "hllc", "br0", False) == 2
    assert T.get_variant(5, "hllc", "local_dd", True) == 1


def test_load_merges_and_ignores_unknown_keys(tmp_path):
    path = str(tmp_path / "t.json")
    with open(path, "w") as f:
        json.dump({"format": "frforge_b200 autotune table", "version": 1, "note": {"a": [1, 2]},
                   "entries": [{"geometry": "affine", "variant": 1, "p": 2, "flux": "hllc", "av": "br0",
                                "ms": 0.5, "extra": "x"}]}, f)
    T.set_variant(4, "rusanov", "br0", False, 0)
    T.load(path)
    assert T.size() == 2 and T.get_variant(2, "hllc", "br0", False) == 1


@pytest.mark.parametrize("text", [
    "", "{", "[]", '{"entries": [{"p": 3}]}', '{"entries": [{"p": 3, "flux": "hllc", "av": "br0", '
    '"geometry": "affine", "variant": 42}]}', '{"entries": [{"p": 3, "flux": "roe", "av": "br0", '
    '"geometry": "affine", "variant": 0}]}', '{"version": 1}',
])
def test_malformed_files_merge_nothing(tmp_path, text):
    path = str(tmp_path / "bad.json")
    with open(path, "w") as f:
        f.write(text)
    T.set_variant(3, "hllc", "br0", False, 1)
    with pytest.raises(ValueError):
        T.load(path)
    assert T.size() == 1 and T.get_variant(3, "hllc", "br0", False) == 1


def test_committed_b200_table_loads():
    if not os.path.exists(T.DEFAULT_TABLE):
        pytest.skip("no committed table")
    assert T.load_default()
    assert T.size() >= 1
    with open(T.DEFAULT_TABLE) as f:
        d = json.load(f)
    for e in d["entries"]:
        assert T.get_variant(e["p"], e["flux"], e["av"], e["geometry"] == "curved") == e["variant"]


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(ValueError):
        T.load(str(tmp_path / "absent.json"))
    assert L.load().frg_autotune_table_size() == 0
