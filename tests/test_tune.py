"""The tuner's cache file (kg_tune_lookup / kg_tune_store): a versioned JSON map of
(GPU, shape class) -> choice, read and written without a GPU."""

import json

import kyto_b200 as K

GPU = "NVIDIA B200/sm_100/148 SMs"
CLS = "knn_filter/n2^20/d50/k14"


def test_store_then_lookup_round_trips(tmp_path):
    path = tmp_path / "sub" / "tune.json"  # the directory is made on the first store
    assert K.tune_lookup(path, GPU, CLS, "kind") is None
    assert K.tune_store(path, GPU, CLS, {"kind": "split", "a_mode": "smem"}, 12.5)
    assert K.tune_lookup(path, GPU, CLS, "kind") == "split"
    assert K.tune_lookup(path, GPU, CLS, "a_mode") == "smem"
    assert K.tune_lookup(path, GPU, CLS, "stages") is None
    assert K.tune_lookup(path, GPU, "knn_filter/n2^21/d50/k14", "kind") is None
    assert K.tune_lookup(path, "another GPU", CLS, "kind") is None
    doc = json.loads(path.read_text())
    assert doc["version"] == 1
    assert doc["entries"] == [{"gpu": GPU, "class": CLS, "ms": 12.5,
                               "choice": {"a_mode": "smem", "kind": "split"}}]


def test_a_second_store_replaces_its_own_entry_and_keeps_the_others(tmp_path):
    path = tmp_path / "tune.json"
    K.tune_store(path, GPU, CLS, {"kind": "fp16", "a_mode": "half"}, 3.0)
    K.tune_store(path, GPU, "other/class", {"kind": "split"}, 4.0)
    K.tune_store(path, GPU, CLS, {"kind": "split", "a_mode": "tmem"}, 2.0)
    doc = json.loads(path.read_text())
    assert len(doc["entries"]) == 2
    assert K.tune_lookup(path, GPU, CLS, "a_mode") == "tmem"
    assert K.tune_lookup(path, GPU, "other/class", "kind") == "split"


def test_another_version_or_a_damaged_file_is_ignored(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"version": 0, "entries": [
        {"gpu": GPU, "class": CLS, "ms": 1, "choice": {"kind": "fp16"}}]}))
    assert K.tune_lookup(path, GPU, CLS, "kind") is None
    # A store rewrites the file under the current version, dropping the old entries.
    assert K.tune_store(path, GPU, "x", {"kind": "split"}, 1.0)
    doc = json.loads(path.read_text())
    assert doc["version"] == 1 and [e["class"] for e in doc["entries"]] == ["x"]
    for damaged in ('{"version": 1, "entries": [', "not json", "", '{"version": 1}',
                    '{"version": 1, "entries": [{"gpu": 3}]}'):
        path.write_text(damaged)
        assert K.tune_lookup(path, GPU, CLS, "kind") is None


def test_strings_with_quotes_and_escapes_survive(tmp_path):
    path = tmp_path / "tune.json"
    gpu = 'a "quoted" GPU \\ name'
    assert K.tune_store(path, gpu, CLS, {"kind": 'sp"lit'}, 0.5)
    assert K.tune_lookup(path, gpu, CLS, "kind") == 'sp"lit'
    assert json.loads(path.read_text())["entries"][0]["gpu"] == gpu


def test_lists_of_different_lengths_are_refused(tmp_path):
    path = str(tmp_path / "t.json").encode()
    assert K.library().kg_tune_store(path, b"g", b"c", b"a;b", b"x", 1.0) == -1
    assert K.library().kg_tune_store(path, b"g", b"c", b"a", b"x;y", 1.0) == -1
    assert not (tmp_path / "t.json").exists()
