"""The autotuner's JSON cache (host logic, no GPU): keys bucket the sizes,
a hit skips the tuning run, a miss runs it once and persists the result,
and an unreadable cache file is an empty cache."""
import json

from cubql_b200 import tuning


def test_cache_key_buckets_sizes():
    a = tuning.cache_key("query", 16, 10_000_000, 10_000_000, gpu="B200")
    assert a == "query|k16|n2^23|q2^23|B200"
    assert tuning.cache_key("query", 16, 9_000_000, 11_000_000, gpu="B200") == a
    assert tuning.cache_key("query", 0, 10_000_000, 10_000_000, gpu="B200") != a


def test_cache_miss_then_hit(tmp_path, monkeypatch):
    monkeypatch.setattr(tuning, "cache_key", lambda kind, k, n, nq, gpu=None: f"{kind}|{k}|{n}|{nq}")
    path = str(tmp_path / "t.json")
    calls = []

    def run():
        calls.append(1)
        return {"makeLeafThreshold": 2, "stackDepth": 64, "blockSize": 128, "queriesPerWarp": 32,
                "buildMs": 1.0, "queryMs": 2.0}
    t1 = tuning._cached("query", 16, 100, 200, run, path)
    t2 = tuning._cached("query", 16, 100, 200, run, path)
    assert len(calls) == 1 and not t1["cached"] and t2["cached"]
    assert t1["stackDepth"] == t2["stackDepth"] == 64
    with open(path) as f:
        assert "query|16|100|200" in json.load(f)
    tuning._cached("query", 16, 100, 200, run, path, retune=True)
    assert len(calls) == 2


def test_unreadable_cache_is_empty(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text("{not json")
    assert tuning._load(str(p)) == {}
    assert tuning._load(str(tmp_path / "missing.json")) == {}
